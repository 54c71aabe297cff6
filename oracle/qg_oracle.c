/*
 * qg_oracle.c -- CPU restatement of the reference's H|psi> path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the GPU engine. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline legs load it. It is
 * pinned against the reference's own code (oracle/_ref, built from the
 * reference headers by oracle/Makefile) and against the committed fixtures in
 * tests/golden/.
 *
 * Each function restates one reference function; the arithmetic grouping of
 * every stencil follows the reference line it cites, and periodic neighbours
 * are read with modular indices instead of the reference's halo copy (the
 * values are identical).
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

typedef struct or_ham_desc {
    int nx, ny, nz;
    double hx, hy, hz;
    int fd_order;
    const double* V;
    int n_atoms;
    const double* atom_pos;
    int n_proj;
    const int* proj_l;
    const double* proj_E;
    const int* cube;
    const double* w_data;
    const long long* w_off;
    int n_lm;
    const double* ylm_data;
    const long long* ylm_off;
} or_ham_desc;

static inline int wrapi(int i, int n) {
    int r = i % n;
    return r < 0 ? r + n : r;
}

#define P(dx, dy, dz) \
    in[(size_t)wrapi(ix + (dx), nx) + (size_t)nx * ((size_t)wrapi(iy + (dy), ny) + (size_t)ny * (size_t)wrapi(iz + (dz), nz))]

/* out += coef * Lap(in), periodic.
 * order 2: Laplasian2nd_halo_f (GridDifference2nd.h:987-1049), "difference first" grouping;
 * order 4: Laplasian4th_halo_f (GridDifference4th.h:478-541), the composed 7-point
 *          stencil (1, -54, 783, -1460)/(24h)^2;
 * order 6: Laplasian6th_halo_f (GridDifference6th.h:373-437), (1, -13.5, 135, -245)/(90h^2);
 * order 8: Laplasian8th_halo_f (GridDifference8th.h:83-149), (-9, 128, -1008, 8064, -14350)/(5040h^2). */
int or_laplacian(int order, int nx, int ny, int nz, double hx, double hy, double hz, double coef,
                 const double* in, double* out) {
    if (order == 2) {
        const double c1x = coef / (hx * hx), c1y = coef / (hy * hy), c1z = coef / (hz * hz);
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    const double c = P(0, 0, 0);
                    const double d = c1x * (P(1, 0, 0) + P(-1, 0, 0) - 2.0 * c)
                                   + c1y * (P(0, 1, 0) + P(0, -1, 0) - 2.0 * c)
                                   + c1z * (P(0, 0, 1) + P(0, 0, -1) - 2.0 * c);
                    out[ix + (size_t)nx * (iy + (size_t)ny * iz)] += d;
                }
        return 0;
    }
    if (order == 4) {
        const double c3x = coef / ((24.0 * hx) * (24.0 * hx));
        const double c3y = coef / ((24.0 * hy) * (24.0 * hy));
        const double c3z = coef / ((24.0 * hz) * (24.0 * hz));
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    const double c = P(0, 0, 0);
                    const double d =
                        c3x * ((P(3, 0, 0) + P(-3, 0, 0)) - 54.0 * (P(2, 0, 0) + P(-2, 0, 0)) + 783.0 * (P(1, 0, 0) + P(-1, 0, 0)) - 1460.0 * c)
                      + c3y * ((P(0, 3, 0) + P(0, -3, 0)) - 54.0 * (P(0, 2, 0) + P(0, -2, 0)) + 783.0 * (P(0, 1, 0) + P(0, -1, 0)) - 1460.0 * c)
                      + c3z * ((P(0, 0, 3) + P(0, 0, -3)) - 54.0 * (P(0, 0, 2) + P(0, 0, -2)) + 783.0 * (P(0, 0, 1) + P(0, 0, -1)) - 1460.0 * c);
                    out[ix + (size_t)nx * (iy + (size_t)ny * iz)] += d;
                }
        return 0;
    }
    if (order == 6) {
        const double c0 = -245.0 * coef * (1.0 / (90.0 * hx * hx) + 1.0 / (90.0 * hy * hy) + 1.0 / (90.0 * hz * hz));
        const double c3x = coef / (90.0 * hx * hx), c2x = -13.5 * coef / (90.0 * hx * hx), c1x = 135.0 * coef / (90.0 * hx * hx);
        const double c3y = coef / (90.0 * hy * hy), c2y = -13.5 * coef / (90.0 * hy * hy), c1y = 135.0 * coef / (90.0 * hy * hy);
        const double c3z = coef / (90.0 * hz * hz), c2z = -13.5 * coef / (90.0 * hz * hz), c1z = 135.0 * coef / (90.0 * hz * hz);
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    double d = c0 * P(0, 0, 0);
                    d += c3x * (P(3, 0, 0) + P(-3, 0, 0)) + c2x * (P(2, 0, 0) + P(-2, 0, 0)) + c1x * (P(1, 0, 0) + P(-1, 0, 0));
                    d += c3y * (P(0, 3, 0) + P(0, -3, 0)) + c2y * (P(0, 2, 0) + P(0, -2, 0)) + c1y * (P(0, 1, 0) + P(0, -1, 0));
                    d += c3z * (P(0, 0, 3) + P(0, 0, -3)) + c2z * (P(0, 0, 2) + P(0, 0, -2)) + c1z * (P(0, 0, 1) + P(0, 0, -1));
                    out[ix + (size_t)nx * (iy + (size_t)ny * iz)] += d;
                }
        return 0;
    }
    if (order == 8) {
        const double c0 = -14350.0 / 5040.0 * coef * (1.0 / (hx * hx) + 1.0 / (hy * hy) + 1.0 / (hz * hz));
        const double c4x = -9.0 * coef / (5040.0 * hx * hx), c3x = 128.0 * coef / (5040.0 * hx * hx);
        const double c2x = -1008.0 * coef / (5040.0 * hx * hx), c1x = 8064.0 * coef / (5040.0 * hx * hx);
        const double c4y = -9.0 * coef / (5040.0 * hy * hy), c3y = 128.0 * coef / (5040.0 * hy * hy);
        const double c2y = -1008.0 * coef / (5040.0 * hy * hy), c1y = 8064.0 * coef / (5040.0 * hy * hy);
        const double c4z = -9.0 * coef / (5040.0 * hz * hz), c3z = 128.0 * coef / (5040.0 * hz * hz);
        const double c2z = -1008.0 * coef / (5040.0 * hz * hz), c1z = 8064.0 * coef / (5040.0 * hz * hz);
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    double d = c0 * P(0, 0, 0);
                    d += c4x * (P(4, 0, 0) + P(-4, 0, 0)) + c3x * (P(3, 0, 0) + P(-3, 0, 0)) + c2x * (P(2, 0, 0) + P(-2, 0, 0)) + c1x * (P(1, 0, 0) + P(-1, 0, 0));
                    d += c4y * (P(0, 4, 0) + P(0, -4, 0)) + c3y * (P(0, 3, 0) + P(0, -3, 0)) + c2y * (P(0, 2, 0) + P(0, -2, 0)) + c1y * (P(0, 1, 0) + P(0, -1, 0));
                    d += c4z * (P(0, 0, 4) + P(0, 0, -4)) + c3z * (P(0, 0, 3) + P(0, 0, -3)) + c2z * (P(0, 0, 2) + P(0, 0, -2)) + c1z * (P(0, 0, 1) + P(0, 0, -1));
                    out[ix + (size_t)nx * (iy + (size_t)ny * iz)] += d;
                }
        return 0;
    }
    return -1;
}

/* One split-complex k-point pass of LaplasianKpoint8th_halo_f
 * (GridDifferenceKpoint8th.h:18-122): out += second-derivative part with
 * c0 including -coef*g^2, out2 += sign1st*2*coef * g.grad(in) (8th-order first
 * derivative (672, -168, 32, -3)/840h), components with |g| < 1e-8 skipped
 * (LaplasianKpoint8th_ddm, :325-368). */
static void kpoint8_pass(int nx, int ny, int nz, double hx, double hy, double hz, double coef,
                         double sign1st, double gx, double gy, double gz, const double* in,
                         double* out, double* out2) {
    const int KX = fabs(gx) >= 1.0e-8, KY = fabs(gy) >= 1.0e-8, KZ = fabs(gz) >= 1.0e-8;
    const double c0 = -14350.0 / 5040.0 * coef * (1.0 / (hx * hx) + 1.0 / (hy * hy) + 1.0 / (hz * hz)) - coef * (gx * gx + gy * gy + gz * gz);
    const double c4x = -9.0 * coef / (5040.0 * hx * hx), c3x = 128.0 * coef / (5040.0 * hx * hx);
    const double c2x = -1008.0 * coef / (5040.0 * hx * hx), c1x = 8064.0 * coef / (5040.0 * hx * hx);
    const double c4y = -9.0 * coef / (5040.0 * hy * hy), c3y = 128.0 * coef / (5040.0 * hy * hy);
    const double c2y = -1008.0 * coef / (5040.0 * hy * hy), c1y = 8064.0 * coef / (5040.0 * hy * hy);
    const double c4z = -9.0 * coef / (5040.0 * hz * hz), c3z = 128.0 * coef / (5040.0 * hz * hz);
    const double c2z = -1008.0 * coef / (5040.0 * hz * hz), c1z = 8064.0 * coef / (5040.0 * hz * hz);
    const double coef2 = sign1st * coef * 2.0;
    const double a1x = 672.0 * coef2 * gx / (840.0 * hx), a2x = -168.0 * coef2 * gx / (840.0 * hx);
    const double a3x = 32.0 * coef2 * gx / (840.0 * hx), a4x = -3.0 * coef2 * gx / (840.0 * hx);
    const double a1y = 672.0 * coef2 * gy / (840.0 * hy), a2y = -168.0 * coef2 * gy / (840.0 * hy);
    const double a3y = 32.0 * coef2 * gy / (840.0 * hy), a4y = -3.0 * coef2 * gy / (840.0 * hy);
    const double a1z = 672.0 * coef2 * gz / (840.0 * hz), a2z = -168.0 * coef2 * gz / (840.0 * hz);
    const double a3z = 32.0 * coef2 * gz / (840.0 * hz), a4z = -3.0 * coef2 * gz / (840.0 * hz);
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                const size_t io = ix + (size_t)nx * (iy + (size_t)ny * iz);
                double d = c0 * P(0, 0, 0);
                d += c4x * (P(4, 0, 0) + P(-4, 0, 0)) + c3x * (P(3, 0, 0) + P(-3, 0, 0)) + c2x * (P(2, 0, 0) + P(-2, 0, 0)) + c1x * (P(1, 0, 0) + P(-1, 0, 0));
                d += c4y * (P(0, 4, 0) + P(0, -4, 0)) + c3y * (P(0, 3, 0) + P(0, -3, 0)) + c2y * (P(0, 2, 0) + P(0, -2, 0)) + c1y * (P(0, 1, 0) + P(0, -1, 0));
                d += c4z * (P(0, 0, 4) + P(0, 0, -4)) + c3z * (P(0, 0, 3) + P(0, 0, -3)) + c2z * (P(0, 0, 2) + P(0, 0, -2)) + c1z * (P(0, 0, 1) + P(0, 0, -1));
                out[io] += d;
                double g = 0.0;
                if (KX) g += a4x * (P(4, 0, 0) - P(-4, 0, 0)) + a3x * (P(3, 0, 0) - P(-3, 0, 0)) + a2x * (P(2, 0, 0) - P(-2, 0, 0)) + a1x * (P(1, 0, 0) - P(-1, 0, 0));
                if (KY) g += a4y * (P(0, 4, 0) - P(0, -4, 0)) + a3y * (P(0, 3, 0) - P(0, -3, 0)) + a2y * (P(0, 2, 0) - P(0, -2, 0)) + a1y * (P(0, 1, 0) - P(0, -1, 0));
                if (KZ) g += a4z * (P(0, 0, 4) - P(0, 0, -4)) + a3z * (P(0, 0, 3) - P(0, 0, -3)) + a2z * (P(0, 0, 2) - P(0, 0, -2)) + a1z * (P(0, 0, 1) - P(0, 0, -1));
                if (KX || KY || KZ) out2[io] += g;
            }
}
/* The 6th-order pass of LaplasianKpoint6th_halo_f (GridDifferenceKpoint6th.h:19-107):
 * c0 = -245 coef sum 1/(90 h^2) - coef g^2, second-derivative (1, -13.5, 135)/(90 h^2),
 * first derivative (45, -9, 1)/(60 h). */
static void kpoint6_pass(int nx, int ny, int nz, double hx, double hy, double hz, double coef,
                         double sign1st, double gx, double gy, double gz, const double* in,
                         double* out, double* out2) {
    const int KX = fabs(gx) >= 1.0e-8, KY = fabs(gy) >= 1.0e-8, KZ = fabs(gz) >= 1.0e-8;
    const double c0 = -245.0 * coef * (1.0 / (90.0 * hx * hx) + 1.0 / (90.0 * hy * hy) + 1.0 / (90.0 * hz * hz)) - coef * (gx * gx + gy * gy + gz * gz);
    const double c3x = coef / (90.0 * hx * hx), c2x = -13.5 * coef / (90.0 * hx * hx), c1x = 135.0 * coef / (90.0 * hx * hx);
    const double c3y = coef / (90.0 * hy * hy), c2y = -13.5 * coef / (90.0 * hy * hy), c1y = 135.0 * coef / (90.0 * hy * hy);
    const double c3z = coef / (90.0 * hz * hz), c2z = -13.5 * coef / (90.0 * hz * hz), c1z = 135.0 * coef / (90.0 * hz * hz);
    const double coef2 = sign1st * coef * 2.0;
    const double a1x = 45.0 * coef2 * gx / (60.0 * hx), a2x = -9.0 * coef2 * gx / (60.0 * hx), a3x = coef2 * gx / (60.0 * hx);
    const double a1y = 45.0 * coef2 * gy / (60.0 * hy), a2y = -9.0 * coef2 * gy / (60.0 * hy), a3y = coef2 * gy / (60.0 * hy);
    const double a1z = 45.0 * coef2 * gz / (60.0 * hz), a2z = -9.0 * coef2 * gz / (60.0 * hz), a3z = coef2 * gz / (60.0 * hz);
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                const size_t io = ix + (size_t)nx * (iy + (size_t)ny * iz);
                double d = c0 * P(0, 0, 0);
                d += c3x * (P(3, 0, 0) + P(-3, 0, 0)) + c2x * (P(2, 0, 0) + P(-2, 0, 0)) + c1x * (P(1, 0, 0) + P(-1, 0, 0));
                d += c3y * (P(0, 3, 0) + P(0, -3, 0)) + c2y * (P(0, 2, 0) + P(0, -2, 0)) + c1y * (P(0, 1, 0) + P(0, -1, 0));
                d += c3z * (P(0, 0, 3) + P(0, 0, -3)) + c2z * (P(0, 0, 2) + P(0, 0, -2)) + c1z * (P(0, 0, 1) + P(0, 0, -1));
                out[io] += d;
                double g = 0.0;
                if (KX) g += a3x * (P(3, 0, 0) - P(-3, 0, 0)) + a2x * (P(2, 0, 0) - P(-2, 0, 0)) + a1x * (P(1, 0, 0) - P(-1, 0, 0));
                if (KY) g += a3y * (P(0, 3, 0) - P(0, -3, 0)) + a2y * (P(0, 2, 0) - P(0, -2, 0)) + a1y * (P(0, 1, 0) - P(0, -1, 0));
                if (KZ) g += a3z * (P(0, 0, 3) - P(0, 0, -3)) + a2z * (P(0, 0, 2) - P(0, 0, -2)) + a1z * (P(0, 0, 1) - P(0, 0, -1));
                if (KX || KY || KZ) out2[io] += g;
            }
}

/* The 2nd-order pass of LaplasianKpoint2nd_halo_f (GridDifferenceKpoint2nd.h:19-92):
 * d = c0 p + c1x (p+x + p-x) + c1y (..) + c1z (..), c0 = -coef sum 2/h^2 - coef g^2,
 * first derivative coef2 g / (2h). */
static void kpoint2_pass(int nx, int ny, int nz, double hx, double hy, double hz, double coef,
                         double sign1st, double gx, double gy, double gz, const double* in,
                         double* out, double* out2) {
    const int KX = fabs(gx) >= 1.0e-8, KY = fabs(gy) >= 1.0e-8, KZ = fabs(gz) >= 1.0e-8;
    const double c0 = -coef * (2.0 / (hx * hx) + 2.0 / (hy * hy) + 2.0 / (hz * hz)) - coef * (gx * gx + gy * gy + gz * gz);
    const double c1x = coef / (hx * hx), c1y = coef / (hy * hy), c1z = coef / (hz * hz);
    const double coef2 = sign1st * coef * 2.0;
    const double a1x = coef2 * gx / (2.0 * hx), a1y = coef2 * gy / (2.0 * hy), a1z = coef2 * gz / (2.0 * hz);
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                const size_t io = ix + (size_t)nx * (iy + (size_t)ny * iz);
                const double d = c0 * P(0, 0, 0) + c1x * (P(1, 0, 0) + P(-1, 0, 0)) + c1y * (P(0, 1, 0) + P(0, -1, 0)) +
                                 c1z * (P(0, 0, 1) + P(0, 0, -1));
                out[io] += d;
                double g = 0.0;
                if (KX) g += a1x * (P(1, 0, 0) - P(-1, 0, 0));
                if (KY) g += a1y * (P(0, 1, 0) - P(0, -1, 0));
                if (KZ) g += a1z * (P(0, 0, 1) - P(0, 0, -1));
                if (KX || KY || KZ) out2[io] += g;
            }
}
#undef P

/* LaplasianKpoint{2nd,6th,8th}_halo (GridDifferenceKpoint2nd.h, 6th.h:109-142,
 * 8th.h:124-157) for order 2, 6 or 8: the real part pass (sign +1) writes out_re and the
 * first-derivative term into out_im, the imaginary part pass (sign -1) writes out_im
 * and the derivative into out_re. Returns -1 for another order. */
int or_laplacian_kpoint(int order, int nx, int ny, int nz, double hx, double hy, double hz, double coef,
                        double gx, double gy, double gz, const double* re, const double* im,
                        double* out_re, double* out_im) {
    switch (order) {
        case 2:
            kpoint2_pass(nx, ny, nz, hx, hy, hz, coef, +1.0, gx, gy, gz, re, out_re, out_im);
            kpoint2_pass(nx, ny, nz, hx, hy, hz, coef, -1.0, gx, gy, gz, im, out_im, out_re);
            return 0;
        case 6:
            kpoint6_pass(nx, ny, nz, hx, hy, hz, coef, +1.0, gx, gy, gz, re, out_re, out_im);
            kpoint6_pass(nx, ny, nz, hx, hy, hz, coef, -1.0, gx, gy, gz, im, out_im, out_re);
            return 0;
        case 8:
            kpoint8_pass(nx, ny, nz, hx, hy, hz, coef, +1.0, gx, gy, gz, re, out_re, out_im);
            kpoint8_pass(nx, ny, nz, hx, hy, hz, coef, -1.0, gx, gy, gz, im, out_im, out_re);
            return 0;
        default: return -1;
    }
}

/* LaplasianKpoint8th_halo (GridDifferenceKpoint8th.h:124-157): the real part
 * pass (sign +1) writes out_re and the first-derivative term into out_im, the
 * imaginary part pass (sign -1) writes out_im and the derivative into out_re. */
int or_laplacian_kpoint8(int nx, int ny, int nz, double hx, double hy, double hz, double coef,
                         double gx, double gy, double gz, const double* re, const double* im,
                         double* out_re, double* out_im) {
    kpoint8_pass(nx, ny, nz, hx, hy, hz, coef, +1.0, gx, gy, gz, re, out_re, out_im);
    kpoint8_pass(nx, ny, nz, hx, hy, hz, coef, -1.0, gx, gy, gz, im, out_im, out_re);
    return 0;
}

/* ProjectionPP (PseudoPotOperator.h:740-772) for one real state:
 * l = 0: c = dV*Y00*sum(w psi); Hp += (E*Y00*c) w          (InnerProd_1S_1R / Add_1S)
 * l > 0: c = dV*sum(w Y psi);   Hp += (E*c) w Y per m      (InnerProd_2S_1R / Add_2S)
 * Periodic images (ForOverlapPeriodic, GridSubgrid.h:267-299) are the cube
 * points mapped back into the grid by modular indices. */
static void nonlocal_one(const or_ham_desc* d, const double* psi, double* Hp) {
    const double coef = d->hx * d->hy * d->hz;
    const double Y00 = 1.0 / sqrt(4.0 * M_PI);
    const int nx = d->nx, ny = d->ny, nz = d->nz;
    for (int a = 0; a < d->n_atoms; ++a) {
        for (int k = 0; k < d->n_proj; ++k) {
            const int l = d->proj_l[k];
            const int* c = d->cube + 6 * ((size_t)a * d->n_proj + k);
            const int bx = c[0], by = c[1], bz = c[2], sx = c[3], sy = c[4], sz = c[5];
            const double* w = d->w_data + d->w_off[(size_t)a * d->n_proj + k];
            const int nm = (l == 0) ? 1 : 2 * l + 1;
            for (int m1 = 0; m1 < nm; ++m1) {
                const double* Y = (l == 0) ? NULL : d->ylm_data + d->ylm_off[(size_t)a * d->n_lm + l * l + m1];
                double sum = 0.0;
                for (int kz = 0; kz < sz; ++kz) {
                    const size_t gz = (size_t)wrapi(bz + kz, nz);
                    for (int ky = 0; ky < sy; ++ky) {
                        const size_t gy = (size_t)wrapi(by + ky, ny);
                        for (int kx = 0; kx < sx; ++kx) {
                            const size_t q = kx + (size_t)sx * (ky + (size_t)sy * kz);
                            const size_t g = (size_t)wrapi(bx + kx, nx) + nx * (gy + ny * gz);
                            sum += (Y ? w[q] * Y[q] : w[q]) * psi[g];
                        }
                    }
                }
                double inner = (l == 0) ? coef * Y00 * sum : coef * sum;
                inner *= d->proj_E[k];
                if (l == 0) inner *= Y00;
                for (int kz = 0; kz < sz; ++kz) {
                    const size_t gz = (size_t)wrapi(bz + kz, nz);
                    for (int ky = 0; ky < sy; ++ky) {
                        const size_t gy = (size_t)wrapi(by + ky, ny);
                        for (int kx = 0; kx < sx; ++kx) {
                            const size_t q = kx + (size_t)sx * (ky + (size_t)sy * kz);
                            const size_t g = (size_t)wrapi(bx + kx, nx) + nx * (gy + ny * gz);
                            Hp[g] += Y ? inner * w[q] * Y[q] : inner * w[q];
                        }
                    }
                }
            }
        }
    }
}

/* mHamiltonianMatrix_ddm (qumasun_mpi.matrix.h:20-43) for ns states:
 * Hp = V psi (mPotentialMatrix_ddm, :158-164); Hp += V_NL psi; Hp += -1/2 Lap psi. */
int or_hamiltonian_apply(const or_ham_desc* d, int ns, const double* X, double* HX) {
    const size_t N = (size_t)d->nx * d->ny * d->nz;
    for (int s = 0; s < ns; ++s) {
        const double* psi = X + (size_t)s * N;
        double* Hp = HX + (size_t)s * N;
        for (size_t i = 0; i < N; ++i) Hp[i] = d->V[i] * psi[i];
        if (d->n_atoms > 0 && d->n_proj > 0) nonlocal_one(d, psi, Hp);
        int rc = or_laplacian(d->fd_order, d->nx, d->ny, d->nz, d->hx, d->hy, d->hz, -0.5, psi, Hp);
        if (rc) return rc;
    }
    return 0;
}

/* Complex k-point Hamiltonian of mHamiltonianMatrix_ddm (qumasun_kpoint.matrix.h:25-50)
 * without the nonlocal term: V on re and im, then the k-point kinetic term.
 * Each state is {re[N], im[N]} contiguous. */
int or_hamiltonian_kpoint_local(const or_ham_desc* d, double gx, double gy, double gz, int ns,
                                const double* X, double* HX) {
    const size_t N = (size_t)d->nx * d->ny * d->nz;
    for (int s = 0; s < ns; ++s) {
        const double* re = X + (size_t)s * 2 * N;
        const double* im = re + N;
        double* ore = HX + (size_t)s * 2 * N;
        double* oim = ore + N;
        for (size_t i = 0; i < N; ++i) { ore[i] = d->V[i] * re[i]; oim[i] = d->V[i] * im[i]; }
        if (or_laplacian_kpoint(d->fd_order, d->nx, d->ny, d->nz, d->hx, d->hy, d->hz, -0.5, gx, gy, gz, re, im, ore,
                                oim) != 0)
            return -1;
    }
    return 0;
}

/* ProjectionPP of PseudoPotIntegrator_kpoint (PseudoPotOperator_kpoint_v2.h:2581-2700)
 * for one {re, im} state. The projector on cube point q of atom a is
 *   P(q) = w_k(q) Y(q) exp(i theta(q)),  theta = gx hx ux + gy hy uy + gz hz uz,
 * u the point's unwrapped grid coordinate (mCreateProjectorRadialOnBlock, :287-420).
 * Contraction without conjugate (mInnerNonlocalPsi_v2, :836-905):
 *   c = dV (Y00 for l = 0) sum_q P(q) psi(g(q));
 * scatter with the conjugate: Hpsi(g(q)) += E (Y00 for l = 0) conj(P(q)) c. */
static void nonlocal_kpoint_one(const or_ham_desc* d, double gx, double gy, double gz, const double* re,
                                const double* im, double* ore, double* oim) {
    const double dV = d->hx * d->hy * d->hz;
    const double Y00 = 1.0 / sqrt(4.0 * M_PI);
    const int nx = d->nx, ny = d->ny, nz = d->nz;
    const double ax = gx * d->hx, ay = gy * d->hy, az = gz * d->hz;
    for (int a = 0; a < d->n_atoms; ++a) {
        for (int k = 0; k < d->n_proj; ++k) {
            const int l = d->proj_l[k];
            const int* c = d->cube + 6 * ((size_t)a * d->n_proj + k);
            const int bx = c[0], by = c[1], bz = c[2], sx = c[3], sy = c[4], sz = c[5];
            const double* w = d->w_data + d->w_off[(size_t)a * d->n_proj + k];
            const int nm = 2 * l + 1;
            for (int m1 = 0; m1 < nm; ++m1) {
                const double* Y = (l == 0) ? NULL : d->ylm_data + d->ylm_off[(size_t)a * d->n_lm + l * l + m1];
                double sr = 0.0, si = 0.0;
                for (int kz = 0; kz < sz; ++kz)
                    for (int ky = 0; ky < sy; ++ky)
                        for (int kx = 0; kx < sx; ++kx) {
                            const size_t q = kx + (size_t)sx * (ky + (size_t)sy * kz);
                            const double th = ax * (double)(bx + kx) + ay * (double)(by + ky) + az * (double)(bz + kz);
                            const double p = Y ? w[q] * Y[q] : w[q];
                            const double pr = p * cos(th), pi = p * sin(th);
                            const size_t g = (size_t)wrapi(bx + kx, nx) +
                                             (size_t)nx * ((size_t)wrapi(by + ky, ny) + (size_t)ny * (size_t)wrapi(bz + kz, nz));
                            sr += pr * re[g] - pi * im[g];
                            si += pi * re[g] + pr * im[g];
                        }
                const double s = (l == 0) ? dV * Y00 * Y00 * d->proj_E[k] : dV * d->proj_E[k];
                const double cr = sr * s, ci = si * s;
                for (int kz = 0; kz < sz; ++kz)
                    for (int ky = 0; ky < sy; ++ky)
                        for (int kx = 0; kx < sx; ++kx) {
                            const size_t q = kx + (size_t)sx * (ky + (size_t)sy * kz);
                            const double th = ax * (double)(bx + kx) + ay * (double)(by + ky) + az * (double)(bz + kz);
                            const double p = Y ? w[q] * Y[q] : w[q];
                            const double pr = p * cos(th), pi = p * sin(th);
                            const size_t g = (size_t)wrapi(bx + kx, nx) +
                                             (size_t)nx * ((size_t)wrapi(by + ky, ny) + (size_t)ny * (size_t)wrapi(bz + kz, nz));
                            ore[g] += pr * cr + pi * ci;
                            oim[g] += pr * ci - pi * cr;
                        }
            }
        }
    }
}

/* Complex k-point Hamiltonian, mHamiltonianMatrix_ddm of QUMASUN_KPOINT
 * (qumasun_kpoint.matrix.h:25-50): V on re and im, the k-point nonlocal term,
 * then the k-point kinetic term of the descriptor's FD order (2, 6 or 8). Each state is {re[N], im[N]} contiguous. */
int or_hamiltonian_kpoint_apply(const or_ham_desc* d, double gx, double gy, double gz, int ns, const double* X,
                                double* HX) {
    const size_t N = (size_t)d->nx * d->ny * d->nz;
    for (int s = 0; s < ns; ++s) {
        const double* re = X + (size_t)s * 2 * N;
        const double* im = re + N;
        double* ore = HX + (size_t)s * 2 * N;
        double* oim = ore + N;
        for (size_t i = 0; i < N; ++i) { ore[i] = d->V[i] * re[i]; oim[i] = d->V[i] * im[i]; }
        if (d->n_atoms > 0 && d->n_proj > 0) nonlocal_kpoint_one(d, gx, gy, gz, re, im, ore, oim);
        if (or_laplacian_kpoint(d->fd_order, d->nx, d->ny, d->nz, d->hx, d->hy, d->hz, -0.5, gx, gy, gz, re, im, ore,
                                oim) != 0)
            return -1;
    }
    return 0;
}
