/*
 * TEST INFRASTRUCTURE -- parity oracle, not part of the product.
 *
 * Plain-C restatement of the vendored NCAR FFTPACK variant that the reference
 * ships in cft_buff.f (complex transforms along z) and rft_buff.f (real
 * transforms along x).  The operation order, the twiddle tables (rotation
 * recurrence for the complex transform, direct cos/sin for the real one) and
 * the truncated constants are kept as the reference has them so that the
 * oracle rounds the way the reference does.  Only radices 2, 3 and 4 are
 * restated: the reference's real transform stops on any other factor
 * (rft_buff.f:308-311, 560-562), and the channel sizes this path serves are
 * 2/3-smooth.  The generic odd-radix passes (cft_buff.f:536-626, 983-1073)
 * are not restated; a length with another prime factor is rejected.
 *
 * Only tests/, the smoke check and the CPU-baseline leg of bench.py use this.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "lh_oracle.h"

/* cft_buff.f:333 / :780 and rft_buff.f:364,616 : 15-digit sqrt(3)/2 */
static const double TAUR = -0.5;
static const double TAUI = 0.866025403784439;
/* rft_buff.f:404 and :658 */
static const double HSQT2 = 0.7071067811865475;
static const double SQRT2 = 1.414213562373095;

/* ------------------------------------------------------------------ */
/* factorisation (cffti1 cft_buff.f:141-163, rffti1 rft_buff.f:133-160) */
static int factorize(int n, const int ntryh[4], int *ifac)
{
    int nl = n, nf = 0, j = 0, ntry = 0;
    for (;;) {
        j++;
        ntry = (j <= 4) ? ntryh[j - 1] : ntry + 2;
        for (;;) {
            int nq = nl / ntry;
            int nr = nl - ntry * nq;
            if (nr != 0) break;
            nf++;
            ifac[nf + 1] = ntry; /* ifac(nf+2) with 1-based ifac */
            nl = nq;
            if (ntry == 2 && nf != 1) {
                for (int i = 2; i <= nf; i++) {
                    int ib = nf - i + 2;
                    ifac[ib + 1] = ifac[ib];
                }
                ifac[2] = 2;
            }
            if (nl == 1) {
                ifac[0] = n;
                ifac[1] = nf;
                return nf;
            }
        }
    }
}

static int radix_ok(const int *ifac)
{
    for (int k = 0; k < ifac[1]; k++) {
        int p = ifac[k + 2];
        if (p != 2 && p != 3 && p != 4) return 0;
    }
    return 1;
}

/* ------------------------------------------------------------------ */
/* complex transform tables: cfti + cffti + cffti1 (cft_buff.f:71-181) */
int lho_cfft_init(lho_cfft *t, int n)
{
    static const int ntryh[4] = {3, 4, 2, 5};
    memset(t, 0, sizeof(*t));
    t->n = n;
    t->dn1 = 1.0 / n;
    if (n < 2 || n > LHO_FFT_MAXN) return -1;
    factorize(n, ntryh, t->ifac);
    if (!radix_ok(t->ifac)) return -2;
    /* rotation recurrence, cft_buff.f:166-179 */
    double tpi = 8.0 * atan(1.0);
    double arg1 = tpi / (double)(float)n;
    double dc = cos(arg1), ds = sin(arg1);
    t->wa[0] = dc;
    t->wa[1] = ds;
    for (int i = 4; i <= 2 * n; i += 2) {
        t->wa[i - 2] = dc * t->wa[i - 4] - ds * t->wa[i - 3];
        t->wa[i - 1] = ds * t->wa[i - 4] + dc * t->wa[i - 3];
    }
    return 0;
}

/*
 * Index helpers for the Fortran arrays of the passes.  All arrays are
 * 1-based in the reference; the macros take 1-based indices.
 *   cc(ido,ip,l1), c1/ch(ido,l1,ip), c2/ch2(idl1,ip)
 */
#define CC(i, j, k) cc[((i) - 1) + ido * (((j) - 1) + ip * ((k) - 1))]
#define C1(i, k, j) c[((i) - 1) + ido * (((k) - 1) + l1 * ((j) - 1))]
#define CH(i, k, j) ch[((i) - 1) + ido * (((k) - 1) + l1 * ((j) - 1))]
#define C2(ik, j) c[((ik) - 1) + idl1 * ((j) - 1)]
#define CH2(ik, j) ch[((ik) - 1) + idl1 * ((j) - 1)]
/* twiddle wa1(l1*m-1), leading dimension ld, column i-2 (1-based) */
#define WA(ld, r, col) wa[((r) - 1) + (ld) * ((col) - 1)]

/*
 * passb2/passf2 (cft_buff.f:279-325, 725-771).  `sgn` = +1 backward,
 * -1 forward; the forward pass differs only in the sign of the twiddle's
 * imaginary part.
 */
static void pass2(int sgn, int ido, int l1, int idl1, double *c, double *ch,
                  const double *wa)
{
    const int ip = 2;
    const double *cc = c;
    for (int k = 1; k <= l1; k++)
        for (int i = 1; i <= ido; i++) {
            CH(i, k, 1) = CC(i, 1, k) + CC(i, 2, k);
            CH(i, k, 2) = CC(i, 1, k) - CC(i, 2, k);
        }
    for (int ik = 1; ik <= idl1; ik++) C2(ik, 1) = CH2(ik, 1);
    for (int k = 1; k <= l1; k++) {
        C1(1, k, 2) = CH(1, k, 2);
        C1(2, k, 2) = CH(2, k, 2);
    }
    if (ido == 2) return;
    for (int k = 1; k <= l1; k++)
        for (int i = 4; i <= ido; i += 2) {
            double wr = WA(l1, l1 - 1, i - 2), wi = WA(l1, l1, i - 2);
            if (sgn > 0) {
                C1(i, k, 2) = wr * CH(i, k, 2) + wi * CH(i - 1, k, 2);
                C1(i - 1, k, 2) = wr * CH(i - 1, k, 2) - wi * CH(i, k, 2);
            } else {
                C1(i, k, 2) = wr * CH(i, k, 2) - wi * CH(i - 1, k, 2);
                C1(i - 1, k, 2) = wr * CH(i - 1, k, 2) + wi * CH(i, k, 2);
            }
        }
}

/* passb3/passf3 (cft_buff.f:329-399, 776-843) */
static void pass3(int sgn, int ido, int l1, int idl1, int ix2, double *c,
                  double *ch, const double *wa)
{
    const int ip = 3;
    const double *cc = c;
    const double taui = sgn > 0 ? TAUI : -TAUI;
    for (int k = 1; k <= l1; k++)
        for (int i = 1; i <= ido; i++) {
            CH(i, k, 1) = CC(i, 1, k);
            CH(i, k, 2) = CC(i, 2, k) + CC(i, 3, k);
            CH(i, k, 3) = CC(i, 2, k) - CC(i, 3, k);
        }
    for (int ik = 1; ik <= idl1; ik++) {
        C2(ik, 1) = CH2(ik, 1) + CH2(ik, 2);
        C2(ik, 2) = CH2(ik, 1) + TAUR * CH2(ik, 2);
        C2(ik, 3) = taui * CH2(ik, 3);
    }
    for (int ik = 2; ik <= idl1; ik += 2) {
        CH2(ik - 1, 2) = C2(ik - 1, 2) - C2(ik, 3);
        CH2(ik - 1, 3) = C2(ik - 1, 2) + C2(ik, 3);
    }
    for (int ik = 2; ik <= idl1; ik += 2) {
        CH2(ik, 2) = C2(ik, 2) + C2(ik - 1, 3);
        CH2(ik, 3) = C2(ik, 2) - C2(ik - 1, 3);
    }
    for (int j = 2; j <= 3; j++)
        for (int k = 1; k <= l1; k++) {
            C1(1, k, j) = CH(1, k, j);
            C1(2, k, j) = CH(2, k, j);
        }
    if (ido == 2) return;
    for (int k = 1; k <= l1; k++)
        for (int i = 4; i <= ido; i += 2) {
            double w1r = WA(l1, l1 - 1, i - 2), w1i = WA(l1, l1, i - 2);
            double w2r = WA(ix2, ix2 - 1, i - 2), w2i = WA(ix2, ix2, i - 2);
            if (sgn > 0) {
                C1(i, k, 2) = w1r * CH(i, k, 2) + w1i * CH(i - 1, k, 2);
                C1(i - 1, k, 2) = w1r * CH(i - 1, k, 2) - w1i * CH(i, k, 2);
                C1(i, k, 3) = w2r * CH(i, k, 3) + w2i * CH(i - 1, k, 3);
                C1(i - 1, k, 3) = w2r * CH(i - 1, k, 3) - w2i * CH(i, k, 3);
            } else {
                C1(i, k, 2) = w1r * CH(i, k, 2) - w1i * CH(i - 1, k, 2);
                C1(i - 1, k, 2) = w1r * CH(i - 1, k, 2) + w1i * CH(i, k, 2);
                C1(i, k, 3) = w2r * CH(i, k, 3) - w2i * CH(i - 1, k, 3);
                C1(i - 1, k, 3) = w2r * CH(i - 1, k, 3) + w2i * CH(i, k, 3);
            }
        }
}

/* passb4/passf4 (cft_buff.f:404-532, 848-978) */
static void pass4(int sgn, int ido, int l1, int idl1, int ix2, int ix3,
                  double *c, double *ch, const double *wa)
{
    const int ip = 4;
    const double *cc = c;
    for (int k = 1; k <= l1; k++) {
        for (int i = 2; i <= ido; i += 2) {
            if (sgn > 0) {
                CH(i - 1, k, 4) = CC(i, 4, k) - CC(i, 2, k);
                CH(i, k, 4) = CC(i - 1, 2, k) - CC(i - 1, 4, k);
            } else {
                CH(i - 1, k, 4) = CC(i, 2, k) - CC(i, 4, k);
                CH(i, k, 4) = CC(i - 1, 4, k) - CC(i - 1, 2, k);
            }
        }
        for (int i = 1; i <= ido; i++) {
            CH(i, k, 2) = CC(i, 1, k) + CC(i, 3, k);
            CH(i, k, 3) = CC(i, 2, k) + CC(i, 4, k);
            CH(i, k, 1) = CC(i, 1, k) - CC(i, 3, k);
        }
    }
    for (int ik = 1; ik <= idl1; ik++) C2(ik, 1) = CH2(ik, 2) + CH2(ik, 3);
    for (int ik = 1; ik <= idl1; ik++) CH2(ik, 3) = CH2(ik, 2) - CH2(ik, 3);
    for (int ik = 1; ik <= idl1; ik++) CH2(ik, 2) = CH2(ik, 1) + CH2(ik, 4);
    for (int ik = 1; ik <= idl1; ik++) CH2(ik, 4) = CH2(ik, 1) - CH2(ik, 4);
    for (int j = 2; j <= 4; j++)
        for (int k = 1; k <= l1; k++) {
            C1(1, k, j) = CH(1, k, j);
            C1(2, k, j) = CH(2, k, j);
        }
    if (ido == 2) return;
    for (int k = 1; k <= l1; k++)
        for (int i = 4; i <= ido; i += 2) {
            double w1r = WA(l1, l1 - 1, i - 2), w1i = WA(l1, l1, i - 2);
            double w2r = WA(ix2, ix2 - 1, i - 2), w2i = WA(ix2, ix2, i - 2);
            double w3r = WA(ix3, ix3 - 1, i - 2), w3i = WA(ix3, ix3, i - 2);
            if (sgn > 0) {
                C1(i, k, 2) = w1r * CH(i, k, 2) + w1i * CH(i - 1, k, 2);
                C1(i - 1, k, 2) = w1r * CH(i - 1, k, 2) - w1i * CH(i, k, 2);
                C1(i, k, 3) = w2r * CH(i, k, 3) + w2i * CH(i - 1, k, 3);
                C1(i - 1, k, 3) = w2r * CH(i - 1, k, 3) - w2i * CH(i, k, 3);
                C1(i, k, 4) = w3r * CH(i, k, 4) + w3i * CH(i - 1, k, 4);
                C1(i - 1, k, 4) = w3r * CH(i - 1, k, 4) - w3i * CH(i, k, 4);
            } else {
                C1(i, k, 2) = w1r * CH(i, k, 2) - w1i * CH(i - 1, k, 2);
                C1(i - 1, k, 2) = w1r * CH(i - 1, k, 2) + w1i * CH(i, k, 2);
                C1(i, k, 3) = w2r * CH(i, k, 3) - w2i * CH(i - 1, k, 3);
                C1(i - 1, k, 3) = w2r * CH(i - 1, k, 3) + w2i * CH(i, k, 3);
                C1(i, k, 4) = w3r * CH(i, k, 4) - w3i * CH(i - 1, k, 4);
                C1(i - 1, k, 4) = w3r * CH(i - 1, k, 4) + w3i * CH(i, k, 4);
            }
        }
}

/*
 * cfftb1 / cfftf1 (cft_buff.f:247-274, 693-720): passes in factor order,
 * every pass writes its result back into c.  `c` holds n complex numbers
 * interleaved; `ch` is 2n doubles of scratch.
 */
void lho_cfft_pass(const lho_cfft *t, int sgn, double *c, double *ch)
{
    int n = t->n;
    if (n == 1) return;
    int nf = t->ifac[1];
    int l1 = 1;
    for (int k1 = 1; k1 <= nf; k1++) {
        int ip = t->ifac[k1 + 1];
        int l2 = ip * l1;
        int ido = n / l2;
        int idot = ido + ido;
        int idl1 = idot * l1;
        if (ip == 4) {
            pass4(sgn, idot, l1, idl1, l1 + l1, l1 + l1 + l1, c, ch, t->wa);
        } else if (ip == 2) {
            pass2(sgn, idot, l1, idl1, c, ch, t->wa);
        } else {
            pass3(sgn, idot, l1, idl1, l1 + l1, c, ch, t->wa);
        }
        l1 = l2;
    }
}

/*
 * cft (cft_buff.f:1-65): m strided complex vectors; iopt < 0 forward
 * (e^{-i}, times 1/n), iopt >= 0 backward (e^{+i}, unscaled).
 * `c` is the real array of the reference; ise and isa are in reals.
 */
void lho_cft(double *c, int ise, int isa, int m, int iopt, const lho_cfft *t,
             double *work)
{
    int n = t->n;
    double *aux = work;          /* contiguous copy, 2n */
    double *ch = work + 2 * n;   /* pass scratch, 2n */
    int j00 = 0;
    for (int k = 0; k < m; k++) {
        int j0 = j00;
        for (int j = 0; j < 2 * n; j += 2) {
            aux[j] = c[j0];
            aux[j + 1] = c[j0 + 1];
            j0 += ise;
        }
        if (iopt < 0) {
            lho_cfft_pass(t, -1, aux, ch);
            j0 = j00;
            for (int j = 0; j < 2 * n; j += 2) {
                c[j0] = t->dn1 * aux[j];
                c[j0 + 1] = t->dn1 * aux[j + 1];
                j0 += ise;
            }
        } else {
            lho_cfft_pass(t, +1, aux, ch);
            j0 = j00;
            for (int j = 0; j < 2 * n; j += 2) {
                c[j0] = aux[j];
                c[j0 + 1] = aux[j + 1];
                j0 += ise;
            }
        }
        j00 += isa;
    }
}

#undef CC
#undef C1
#undef CH
#undef C2
#undef CH2

/* ------------------------------------------------------------------ */
/* real transform tables: rfti + rffti + rffti1 (rft_buff.f:1-190)     */
int lho_rfft_init(lho_rfft *t, int n)
{
    static const int ntryh[4] = {4, 2, 3, 5};
    memset(t, 0, sizeof(*t));
    t->n = n;
    t->dn1 = 1.0 / n;
    if (n < 2 || n > LHO_FFT_MAXN || (n & 1)) return -1;
    factorize(n, ntryh, t->ifac);
    if (!radix_ok(t->ifac)) return -2;
    double tpi = 2.0 * atan2(0.0, -1.0);
    double argh = tpi / (double)(float)n;
    int is = 0, nf = t->ifac[1], l1 = 1;
    for (int k1 = 1; k1 <= nf - 1; k1++) {
        int ip = t->ifac[k1 + 1];
        int ld = 0, l2 = l1 * ip, ido = n / l2;
        for (int j = 1; j <= ip - 1; j++) {
            ld += l1;
            int i = is;
            double argld = (double)(float)ld * argh;
            double fi = 0.0;
            for (int ii = 3; ii <= ido; ii += 2) {
                i += 2;
                fi += 1.0;
                double arg = fi * argld;
                t->wa[i - 2] = cos(arg);
                t->wa[i - 1] = sin(arg);
            }
            is += ido;
        }
        l1 = l2;
    }
    return 0;
}

/* radf2 (rft_buff.f:326-353); arrays cc(ido,l1,2) ch(ido,2,l1) */
#define RCC(i, k, j) cc[((i) - 1) + ido * (((k) - 1) + l1 * ((j) - 1))]
#define RCH(i, j, k) ch[((i) - 1) + ido * (((j) - 1) + IP * ((k) - 1))]
static void radf2(int ido, int l1, const double *cc, double *ch,
                  const double *wa1)
{
    const int IP = 2;
    for (int k = 1; k <= l1; k++) {
        RCH(1, 1, k) = RCC(1, k, 1) + RCC(1, k, 2);
        RCH(ido, 2, k) = RCC(1, k, 1) - RCC(1, k, 2);
    }
    if (ido < 2) return;
    if (ido > 2) {
        int idp2 = ido + 2;
        for (int k = 1; k <= l1; k++)
            for (int i = 3; i <= ido; i += 2) {
                int ic = idp2 - i;
                double tr2 = wa1[i - 3] * RCC(i - 1, k, 2) + wa1[i - 2] * RCC(i, k, 2);
                double ti2 = wa1[i - 3] * RCC(i, k, 2) - wa1[i - 2] * RCC(i - 1, k, 2);
                RCH(i, 1, k) = RCC(i, k, 1) + ti2;
                RCH(ic, 2, k) = ti2 - RCC(i, k, 1);
                RCH(i - 1, 1, k) = RCC(i - 1, k, 1) + tr2;
                RCH(ic - 1, 2, k) = RCC(i - 1, k, 1) - tr2;
            }
        if (ido % 2 == 1) return;
    }
    for (int k = 1; k <= l1; k++) {
        RCH(1, 2, k) = -RCC(ido, k, 2);
        RCH(ido, 1, k) = RCC(ido, k, 1);
    }
}

/* radf3 (rft_buff.f:358-398) */
static void radf3(int ido, int l1, const double *cc, double *ch,
                  const double *wa1, const double *wa2)
{
    const int IP = 3;
    for (int k = 1; k <= l1; k++) {
        double cr2 = RCC(1, k, 2) + RCC(1, k, 3);
        RCH(1, 1, k) = RCC(1, k, 1) + cr2;
        RCH(1, 3, k) = TAUI * (RCC(1, k, 3) - RCC(1, k, 2));
        RCH(ido, 2, k) = RCC(1, k, 1) + TAUR * cr2;
    }
    if (ido == 1) return;
    int idp2 = ido + 2;
    for (int k = 1; k <= l1; k++)
        for (int i = 3; i <= ido; i += 2) {
            int ic = idp2 - i;
            double dr2 = wa1[i - 3] * RCC(i - 1, k, 2) + wa1[i - 2] * RCC(i, k, 2);
            double di2 = wa1[i - 3] * RCC(i, k, 2) - wa1[i - 2] * RCC(i - 1, k, 2);
            double dr3 = wa2[i - 3] * RCC(i - 1, k, 3) + wa2[i - 2] * RCC(i, k, 3);
            double di3 = wa2[i - 3] * RCC(i, k, 3) - wa2[i - 2] * RCC(i - 1, k, 3);
            double cr2 = dr2 + dr3;
            double ci2 = di2 + di3;
            RCH(i - 1, 1, k) = RCC(i - 1, k, 1) + cr2;
            RCH(i, 1, k) = RCC(i, k, 1) + ci2;
            double tr2 = RCC(i - 1, k, 1) + TAUR * cr2;
            double ti2 = RCC(i, k, 1) + TAUR * ci2;
            double tr3 = TAUI * (di2 - di3);
            double ti3 = TAUI * (dr3 - dr2);
            RCH(i - 1, 3, k) = tr2 + tr3;
            RCH(ic - 1, 2, k) = tr2 - tr3;
            RCH(i, 3, k) = ti2 + ti3;
            RCH(ic, 2, k) = ti3 - ti2;
        }
}

/* radf4 (rft_buff.f:403-453) */
static void radf4(int ido, int l1, const double *cc, double *ch,
                  const double *wa1, const double *wa2, const double *wa3)
{
    const int IP = 4;
    for (int k = 1; k <= l1; k++) {
        double tr1 = RCC(1, k, 2) + RCC(1, k, 4);
        double tr2 = RCC(1, k, 1) + RCC(1, k, 3);
        RCH(1, 1, k) = tr1 + tr2;
        RCH(ido, 4, k) = tr2 - tr1;
        RCH(ido, 2, k) = RCC(1, k, 1) - RCC(1, k, 3);
        RCH(1, 3, k) = RCC(1, k, 4) - RCC(1, k, 2);
    }
    if (ido < 2) return;
    if (ido > 2) {
        int idp2 = ido + 2;
        for (int k = 1; k <= l1; k++)
            for (int i = 3; i <= ido; i += 2) {
                int ic = idp2 - i;
                double cr2 = wa1[i - 3] * RCC(i - 1, k, 2) + wa1[i - 2] * RCC(i, k, 2);
                double ci2 = wa1[i - 3] * RCC(i, k, 2) - wa1[i - 2] * RCC(i - 1, k, 2);
                double cr3 = wa2[i - 3] * RCC(i - 1, k, 3) + wa2[i - 2] * RCC(i, k, 3);
                double ci3 = wa2[i - 3] * RCC(i, k, 3) - wa2[i - 2] * RCC(i - 1, k, 3);
                double cr4 = wa3[i - 3] * RCC(i - 1, k, 4) + wa3[i - 2] * RCC(i, k, 4);
                double ci4 = wa3[i - 3] * RCC(i, k, 4) - wa3[i - 2] * RCC(i - 1, k, 4);
                double tr1 = cr2 + cr4;
                double tr4 = cr4 - cr2;
                double ti1 = ci2 + ci4;
                double ti4 = ci2 - ci4;
                double ti2 = RCC(i, k, 1) + ci3;
                double ti3 = RCC(i, k, 1) - ci3;
                double tr2 = RCC(i - 1, k, 1) + cr3;
                double tr3 = RCC(i - 1, k, 1) - cr3;
                RCH(i - 1, 1, k) = tr1 + tr2;
                RCH(ic - 1, 4, k) = tr2 - tr1;
                RCH(i, 1, k) = ti1 + ti2;
                RCH(ic, 4, k) = ti1 - ti2;
                RCH(i - 1, 3, k) = ti4 + tr3;
                RCH(ic - 1, 2, k) = tr3 - ti4;
                RCH(i, 3, k) = tr4 + ti3;
                RCH(ic, 2, k) = tr4 - ti3;
            }
        if (ido % 2 == 1) return;
    }
    for (int k = 1; k <= l1; k++) {
        double ti1 = -HSQT2 * (RCC(ido, k, 2) + RCC(ido, k, 4));
        double tr1 = HSQT2 * (RCC(ido, k, 2) - RCC(ido, k, 4));
        RCH(ido, 1, k) = tr1 + RCC(ido, k, 1);
        RCH(ido, 3, k) = RCC(ido, k, 1) - tr1;
        RCH(1, 2, k) = ti1 - RCC(ido, k, 3);
        RCH(1, 4, k) = ti1 + RCC(ido, k, 3);
    }
}
#undef RCC
#undef RCH

/* radb*: arrays cc(ido,IP,l1) ch(ido,l1,IP) */
#define BCC(i, j, k) cc[((i) - 1) + ido * (((j) - 1) + IP * ((k) - 1))]
#define BCH(i, k, j) ch[((i) - 1) + ido * (((k) - 1) + l1 * ((j) - 1))]
/* radb2 (rft_buff.f:580-608) */
static void radb2(int ido, int l1, const double *cc, double *ch,
                  const double *wa1)
{
    const int IP = 2;
    for (int k = 1; k <= l1; k++) {
        BCH(1, k, 1) = BCC(1, 1, k) + BCC(ido, 2, k);
        BCH(1, k, 2) = BCC(1, 1, k) - BCC(ido, 2, k);
    }
    if (ido < 2) return;
    if (ido > 2) {
        int idp2 = ido + 2;
        for (int k = 1; k <= l1; k++)
            for (int i = 3; i <= ido; i += 2) {
                int ic = idp2 - i;
                BCH(i - 1, k, 1) = BCC(i - 1, 1, k) + BCC(ic - 1, 2, k);
                double tr2 = BCC(i - 1, 1, k) - BCC(ic - 1, 2, k);
                BCH(i, k, 1) = BCC(i, 1, k) - BCC(ic, 2, k);
                double ti2 = BCC(i, 1, k) + BCC(ic, 2, k);
                BCH(i - 1, k, 2) = wa1[i - 3] * tr2 - wa1[i - 2] * ti2;
                BCH(i, k, 2) = wa1[i - 3] * ti2 + wa1[i - 2] * tr2;
            }
        if (ido % 2 == 1) return;
    }
    for (int k = 1; k <= l1; k++) {
        BCH(ido, k, 1) = BCC(ido, 1, k) + BCC(ido, 1, k);
        BCH(ido, k, 2) = -(BCC(1, 2, k) + BCC(1, 2, k));
    }
}

/* radb3 (rft_buff.f:613-654) */
static void radb3(int ido, int l1, const double *cc, double *ch,
                  const double *wa1, const double *wa2)
{
    const int IP = 3;
    for (int k = 1; k <= l1; k++) {
        double tr2 = BCC(ido, 2, k) + BCC(ido, 2, k);
        double cr2 = BCC(1, 1, k) + TAUR * tr2;
        BCH(1, k, 1) = BCC(1, 1, k) + tr2;
        double ci3 = TAUI * (BCC(1, 3, k) + BCC(1, 3, k));
        BCH(1, k, 2) = cr2 - ci3;
        BCH(1, k, 3) = cr2 + ci3;
    }
    if (ido == 1) return;
    int idp2 = ido + 2;
    for (int k = 1; k <= l1; k++)
        for (int i = 3; i <= ido; i += 2) {
            int ic = idp2 - i;
            double tr2 = BCC(i - 1, 3, k) + BCC(ic - 1, 2, k);
            double cr2 = BCC(i - 1, 1, k) + TAUR * tr2;
            BCH(i - 1, k, 1) = BCC(i - 1, 1, k) + tr2;
            double ti2 = BCC(i, 3, k) - BCC(ic, 2, k);
            double ci2 = BCC(i, 1, k) + TAUR * ti2;
            BCH(i, k, 1) = BCC(i, 1, k) + ti2;
            double cr3 = TAUI * (BCC(i - 1, 3, k) - BCC(ic - 1, 2, k));
            double ci3 = TAUI * (BCC(i, 3, k) + BCC(ic, 2, k));
            double dr2 = cr2 - ci3;
            double dr3 = cr2 + ci3;
            double di2 = ci2 + cr3;
            double di3 = ci2 - cr3;
            BCH(i - 1, k, 2) = wa1[i - 3] * dr2 - wa1[i - 2] * di2;
            BCH(i, k, 2) = wa1[i - 3] * di2 + wa1[i - 2] * dr2;
            BCH(i - 1, k, 3) = wa2[i - 3] * dr3 - wa2[i - 2] * di3;
            BCH(i, k, 3) = wa2[i - 3] * di3 + wa2[i - 2] * dr3;
        }
}

/* radb4 (rft_buff.f:659-711) */
static void radb4(int ido, int l1, const double *cc, double *ch,
                  const double *wa1, const double *wa2, const double *wa3)
{
    const int IP = 4;
    for (int k = 1; k <= l1; k++) {
        double tr1 = BCC(1, 1, k) - BCC(ido, 4, k);
        double tr2 = BCC(1, 1, k) + BCC(ido, 4, k);
        double tr3 = BCC(ido, 2, k) + BCC(ido, 2, k);
        double tr4 = BCC(1, 3, k) + BCC(1, 3, k);
        BCH(1, k, 1) = tr2 + tr3;
        BCH(1, k, 2) = tr1 - tr4;
        BCH(1, k, 3) = tr2 - tr3;
        BCH(1, k, 4) = tr1 + tr4;
    }
    if (ido < 2) return;
    if (ido > 2) {
        int idp2 = ido + 2;
        for (int k = 1; k <= l1; k++)
            for (int i = 3; i <= ido; i += 2) {
                int ic = idp2 - i;
                double ti1 = BCC(i, 1, k) + BCC(ic, 4, k);
                double ti2 = BCC(i, 1, k) - BCC(ic, 4, k);
                double ti3 = BCC(i, 3, k) - BCC(ic, 2, k);
                double tr4 = BCC(i, 3, k) + BCC(ic, 2, k);
                double tr1 = BCC(i - 1, 1, k) - BCC(ic - 1, 4, k);
                double tr2 = BCC(i - 1, 1, k) + BCC(ic - 1, 4, k);
                double ti4 = BCC(i - 1, 3, k) - BCC(ic - 1, 2, k);
                double tr3 = BCC(i - 1, 3, k) + BCC(ic - 1, 2, k);
                BCH(i - 1, k, 1) = tr2 + tr3;
                double cr3 = tr2 - tr3;
                BCH(i, k, 1) = ti2 + ti3;
                double ci3 = ti2 - ti3;
                double cr2 = tr1 - tr4;
                double cr4 = tr1 + tr4;
                double ci2 = ti1 + ti4;
                double ci4 = ti1 - ti4;
                BCH(i - 1, k, 2) = wa1[i - 3] * cr2 - wa1[i - 2] * ci2;
                BCH(i, k, 2) = wa1[i - 3] * ci2 + wa1[i - 2] * cr2;
                BCH(i - 1, k, 3) = wa2[i - 3] * cr3 - wa2[i - 2] * ci3;
                BCH(i, k, 3) = wa2[i - 3] * ci3 + wa2[i - 2] * cr3;
                BCH(i - 1, k, 4) = wa3[i - 3] * cr4 - wa3[i - 2] * ci4;
                BCH(i, k, 4) = wa3[i - 3] * ci4 + wa3[i - 2] * cr4;
            }
        if (ido % 2 == 1) return;
    }
    for (int k = 1; k <= l1; k++) {
        double ti1 = BCC(1, 2, k) + BCC(1, 4, k);
        double ti2 = BCC(1, 4, k) - BCC(1, 2, k);
        double tr1 = BCC(ido, 1, k) - BCC(ido, 3, k);
        double tr2 = BCC(ido, 1, k) + BCC(ido, 3, k);
        BCH(ido, k, 1) = tr2 + tr2;
        BCH(ido, k, 2) = SQRT2 * (tr1 - ti1);
        BCH(ido, k, 3) = ti2 + ti2;
        BCH(ido, k, 4) = -SQRT2 * (tr1 + ti1);
    }
}
#undef BCC
#undef BCH

/* rfftf1 (rft_buff.f:267-323): factors in reverse order, ping-pong c/ch */
void lho_rfftf(const lho_rfft *t, double *c, double *ch)
{
    int n = t->n, nf = t->ifac[1];
    int na = 1, l2 = n, iw = n;
    for (int k1 = 1; k1 <= nf; k1++) {
        int kh = nf - k1;
        int ip = t->ifac[kh + 2];
        int l1 = l2 / ip;
        int ido = n / l2;
        iw = iw - (ip - 1) * ido;
        na = 1 - na;
        const double *w1 = t->wa + (iw - 1);
        const double *src = na == 0 ? c : ch;
        double *dst = na == 0 ? ch : c;
        if (ip == 4) {
            radf4(ido, l1, src, dst, w1, w1 + ido, w1 + 2 * ido);
        } else if (ip == 2) {
            radf2(ido, l1, src, dst, w1);
        } else {
            radf3(ido, l1, src, dst, w1, w1 + ido);
        }
        l2 = l1;
    }
    if (na == 0) memcpy(c, ch, sizeof(double) * n);
}

/* rfftb1 (rft_buff.f:522-575) */
void lho_rfftb(const lho_rfft *t, double *c, double *ch)
{
    int n = t->n, nf = t->ifac[1];
    int na = 1, l1 = 1, iw = 1;
    for (int k1 = 1; k1 <= nf; k1++) {
        int ip = t->ifac[k1 + 1];
        int l2 = ip * l1;
        int ido = n / l2;
        na = 1 - na;
        const double *w1 = t->wa + (iw - 1);
        const double *src = na == 0 ? c : ch;
        double *dst = na == 0 ? ch : c;
        if (ip == 4) {
            radb4(ido, l1, src, dst, w1, w1 + ido, w1 + 2 * ido);
        } else if (ip == 2) {
            radb2(ido, l1, src, dst, w1);
        } else {
            radb3(ido, l1, src, dst, w1, w1 + ido);
        }
        l1 = l2;
        iw = iw + (ip - 1) * ido;
    }
    if (na == 0) memcpy(c, ch, sizeof(double) * n);
}

/*
 * rft (rft_buff.f:24-86): m real rows of stride isa.  Forward: transform,
 * shift by one slot, scale by 1/n, zero Im(0) and Im(n/2).  Inverse: drop
 * Im(0) by shifting down one slot, then transform.
 */
void lho_rft(double *c, int isa, int m, int iopt, const lho_rfft *t,
             double *work)
{
    int nn = t->n;
    if (iopt < 0) {
        for (int j = 0; j < m; j++) lho_rfftf(t, c + (size_t)j * isa, work);
        for (int j = 0; j < m; j++) {
            double *r = c + (size_t)j * isa;
            for (int i = nn; i >= 2; i--) r[i] = t->dn1 * r[i - 1];
            r[0] = t->dn1 * r[0];
            r[nn + 1] = 0.0;
            r[1] = 0.0;
        }
    } else {
        for (int j = 0; j < m; j++) {
            double *r = c + (size_t)j * isa;
            for (int i = 2; i <= nn; i++) r[i - 1] = r[i];
        }
        for (int j = 0; j < m; j++) lho_rfftb(t, c + (size_t)j * isa, work);
    }
}
