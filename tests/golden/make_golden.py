"""Regenerate the committed golden fixtures from the reference's own data.

Reads the reference's spectral input files (Fortran sequential unformatted,
written by record_out, FOU3D.f90:2066-2165) from the reference tree and
stores, as compressed numpy archives:

* ``grid_ny153_dyq10_p5.npz`` -- yu, yv, dthdyu, dthdyv from the file headers
  (record 3 of each file), the grid known-answer for ygrid (start.f90:665-806).
* ``ref_ic_0032x0032x0153.npz`` -- u1, u2, u3, p of the 32x32x153 initial
  condition exactly as read_in loads it at one MPI rank (start.f90:1545-1997):
  u1/u3 planes 0..nyu, u2 planes 0..nyv+1, p planes 1..nyu, complex per
  column [column, j]; the top ghost plane of u1/u3 is left zero as read_in
  leaves it.  Header scalars t, Re, alp, bet, mpgx, iter are kept too.
* ``ref_turb_0128x0128x0153.npz`` -- the same for the reference's developed
  turbulent 128x128x153 field at t = 945.5 (``*_0128x0128x0153_t09455.dat``).
  At ~81 MB it is not committed (``.gitignore`` lists it): this script makes
  it in a checkout that has the reference tree beside it, and the test that
  steps it skips, naming this script, where the file is absent.

Usage:  python tests/golden/make_golden.py /path/to/reference
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402


def main(ref: str) -> None:
    inp = os.path.join(ref, "input")
    tag = "_0032x0032x0153_t00000.dat"
    fu = O.read_dat(os.path.join(inp, "u1" + tag))
    fv = O.read_dat(os.path.join(inp, "u2" + tag))
    np.savez_compressed(os.path.join(HERE, "grid_ny153_dyq10_p5.npz"),
                        yu=fu.y, yv=fv.y, dthdyu=fu.dthdy, dthdyv=fv.dthdy)
    nyu, nyv = 152, 151
    u1, u2, u3, p, f1 = O.read_in_np1(inp, tag, 32, 32, nyu, nyv)
    np.savez_compressed(os.path.join(HERE, "ref_ic_0032x0032x0153.npz"),
                        u1=u1, u2=u2, u3=u3, p=p,
                        t=f1.t, Re=f1.Re, alp=f1.alp, bet=f1.bet, mpgx=f1.mpgx, iter=f1.iter)
    # the 128x128 turbulent field shares the grid
    f128 = O.read_dat(os.path.join(inp, "u1_0128x0128x0153_t09455.dat"))
    assert np.array_equal(f128.y, fu.y)
    u1, u2, u3, p, f1 = O.read_in_np1(inp, "_0128x0128x0153_t09455.dat", 128, 128, nyu, nyv)
    np.savez(os.path.join(HERE, "ref_turb_0128x0128x0153.npz"),
             u1=u1, u2=u2, u3=u3, p=p,
             t=f1.t, Re=f1.Re, alp=f1.alp, bet=f1.bet, mpgx=f1.mpgx, iter=f1.iter)
    print("wrote golden fixtures to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
