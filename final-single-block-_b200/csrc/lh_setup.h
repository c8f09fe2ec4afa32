// Host-side set-up of one channel instance: the part of the reference's
// start() (start.f90:53-662) that the time step consumes -- the y grid and
// its finite-difference metrics (ygrid, :665-806), wavenumbers (def_k,
// :809-902), grid weights (:518-537), dtv (:476), the pressure matrix
// factors (LU_buildP/LU_decP, tridLU_3D.f90:224-297, 366-407) -- plus the
// FFT twiddle tables and radix plans of the device transforms.
#pragma once

#include <string>
#include <vector>

#include "lh_gpu.h"

namespace lh {

struct HostSetup {
    int Nx = 0, Nz = 0, Mx = 0, Mz = 0, nxh = 0, nc = 0, nyu = 0, nyv = 0;
    std::vector<double> yu, yv, dthdyu, dthdyv, dyu2i, dyv2i;  // dy*2i as [3*j + r]
    std::vector<double> kx, kz, k2x, k2z;                      // kx[i], kz[kr]
    double gw1 = 0, gw2 = 0, gwbc = 0, gwi1 = 0, gwi2 = 0, dtv = 0, ddthetavi = 1.0;
    std::vector<double> DG1, DG2, DG3;                         // DG1[j], DG2/3[(j-1)*nc + col]
    std::vector<double> twz, twx;                              // (re, im) pairs
    std::vector<int> radz, radx;
};

// Validates the description and fills the set-up; returns an empty string
// on success or the reason for rejection.
std::string build_setup(const lh_grid_desc &d, HostSetup &s);

// Radix plans (FFTPACK's factor orders, radices 2, 3, 4 only) and twiddle
// tables exp(+2 pi i t / n), t < n, of the device transforms: complex z
// transforms as cft, real x transforms as rft.  false when n has another
// prime factor.
bool cft_radices(int n, std::vector<int> &rad);
bool rft_radices(int n, std::vector<int> &rad);
void cft_table(int n, std::vector<double> &tw);
void rft_table(int n, std::vector<double> &tw);

// Flow rate of the (0,0) mode of a column-layout u1 (flowrateIm,
// littleharsh.f90:473-492).
double flowrate_host(const HostSetup &s, const double *u1col);

}  // namespace lh
