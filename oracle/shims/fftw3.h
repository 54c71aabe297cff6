/*
 * fftw3.h stand-in for the oracle harness (test infrastructure only).
 *
 * FFTW is not installed here. The reference's Poisson solver (poisson_fft.h via
 * wrap_fft.h) and the TD/k-point class headers (fftw_executor.h) call a handful
 * of FFTW entry points; this header implements them as plain discrete Fourier
 * transforms, one axis after another, straight from the definition
 *   out[k] = sum_j in[j] exp(sign * 2 pi i j k / n),  sign = -1 forward, +1 backward,
 * unnormalised like FFTW. Arrays are row-major (the last dimension fastest), as in
 * fftw_plan_dft_3d(n0, n1, n2, ...). O(n) work per output element per axis: meant
 * for the small grids of the oracle checks, not for speed.
 */
#pragma once
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

typedef double fftw_complex[2];

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

struct qg_fftw_plan_s {
    int n[3];
    int sign;
    int kind;  // 0: complex to complex, 1: real to complex (half spectrum), 2: complex (half) to real
    void* in;
    void* out;
};
typedef qg_fftw_plan_s* fftw_plan;

namespace qg_fftw {

// In-place 1-D DFTs along one axis of a row-major n0 x n1 x n2 complex array.
inline void dft_axis(std::complex<double>* a, const int n[3], int axis, int sign) {
    const int len = n[axis];
    long long stride = 1;
    for (int d = 2; d > axis; --d) stride *= n[d];
    const long long total = (long long)n[0] * n[1] * n[2];
    const long long outer = total / (len * stride);
    std::vector<std::complex<double>> tw(len), tmp(len);
    const double PI = 3.14159265358979323846;
    for (int m = 0; m < len; ++m) tw[m] = std::polar(1.0, sign * 2.0 * PI * (double)m / (double)len);
    for (long long o = 0; o < outer; ++o)
        for (long long s = 0; s < stride; ++s) {
            std::complex<double>* base = a + o * len * stride + s;
            for (int k = 0; k < len; ++k) {
                std::complex<double> acc = 0.0;
                for (int j = 0; j < len; ++j) acc += base[(long long)j * stride] * tw[(long long)j * k % len];
                tmp[k] = acc;
            }
            for (int k = 0; k < len; ++k) base[(long long)k * stride] = tmp[k];
        }
}

inline void dft3(std::complex<double>* a, const int n[3], int sign) {
    for (int axis = 2; axis >= 0; --axis) dft_axis(a, n, axis, sign);
}

}  // namespace qg_fftw

inline fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign,
                                  unsigned) {
    return new qg_fftw_plan_s{{n0, n1, n2}, sign, 0, in, out};
}

inline fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out, unsigned) {
    return new qg_fftw_plan_s{{n0, n1, n2}, -1, 1, in, out};
}

inline fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out, unsigned) {
    return new qg_fftw_plan_s{{n0, n1, n2}, +1, 2, in, out};
}

inline void fftw_execute(const fftw_plan p) {
    const long long total = (long long)p->n[0] * p->n[1] * p->n[2];
    const int nh = p->n[2] / 2 + 1;
    std::vector<std::complex<double>> a(total);
    if (p->kind == 0) {
        const fftw_complex* in = static_cast<const fftw_complex*>(p->in);
        for (long long i = 0; i < total; ++i) a[i] = {in[i][0], in[i][1]};
        qg_fftw::dft3(a.data(), p->n, p->sign);
        fftw_complex* out = static_cast<fftw_complex*>(p->out);
        for (long long i = 0; i < total; ++i) { out[i][0] = a[i].real(); out[i][1] = a[i].imag(); }
    } else if (p->kind == 1) {
        const double* in = static_cast<const double*>(p->in);
        for (long long i = 0; i < total; ++i) a[i] = {in[i], 0.0};
        qg_fftw::dft3(a.data(), p->n, -1);
        fftw_complex* out = static_cast<fftw_complex*>(p->out);
        for (long long r = 0; r < total / p->n[2]; ++r)
            for (int k = 0; k < nh; ++k) {
                out[r * nh + k][0] = a[r * p->n[2] + k].real();
                out[r * nh + k][1] = a[r * p->n[2] + k].imag();
            }
    } else {
        // half spectrum -> full Hermitian spectrum -> real output
        const fftw_complex* in = static_cast<const fftw_complex*>(p->in);
        const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
        for (int i0 = 0; i0 < n0; ++i0)
            for (int i1 = 0; i1 < n1; ++i1)
                for (int k = 0; k < n2; ++k) {
                    std::complex<double> v;
                    if (k < nh) {
                        const long long q = ((long long)i0 * n1 + i1) * nh + k;
                        v = {in[q][0], in[q][1]};
                    } else {
                        const int j0 = (n0 - i0) % n0, j1 = (n1 - i1) % n1, jk = n2 - k;
                        const long long q = ((long long)j0 * n1 + j1) * nh + jk;
                        v = {in[q][0], -in[q][1]};
                    }
                    a[((long long)i0 * n1 + i1) * n2 + k] = v;
                }
        qg_fftw::dft3(a.data(), p->n, +1);
        double* out = static_cast<double*>(p->out);
        for (long long i = 0; i < total; ++i) out[i] = a[i].real();
    }
}

inline void fftw_destroy_plan(fftw_plan p) { delete p; }
inline void* fftw_malloc(size_t bytes) { return std::malloc(bytes); }
inline void fftw_free(void* p) { std::free(p); }
