// Learned LOBPCG preconditioner: a 4-layer periodic 3D convolutional network
//   in  = [r / rms(r), V / vscale]                         (2 channels)
//   h1  = relu(conv3(in)), h2 = relu(conv3(h1)), h3 = relu(conv3(h2))   (16 channels each)
//   out = conv3(h3)                                       (1 channel)
// applied as w = T r + rms(r) * out, T the kinetic preconditioner (precond.cu), so
// the network learns a correction to the plain preconditioner and an untrained
// (zero last layer) network leaves it unchanged. 3^3 kernels, circular padding
// (the grid is periodic), BF16 weights and activations, FP32 accumulation; about
// 15.1k multiply-adds per voxel, as the network the engine was specified with.
//
// Kernels (CUDA cores, one thread per voxel of an 8 x 8 x 4 tile):
//   k_conv_fwd     out[co][v] = b[co] + sum_ci sum_tap W[co][ci][tap] in[ci][v + off(tap)];
//                  the input tile (+ 1-voxel periodic halo) of one channel and that
//                  channel's weights, stored [tap][co], sit in shared memory;
//   backward data  the same kernel with the weights transposed and the taps flipped
//                  (transposed convolution = convolution on a periodic grid), times
//                  the ReLU mask of the layer below;
//   k_conv_wgrad   dW[co][ci][tap] = sum_v dout[co][v] in[ci][v + off(tap)] per tile,
//                  one thread per (ci, tap) holding all co, tile partials summed in a
//                  fixed order (deterministic);
//   k_adam         Adam on FP32 master weights, BF16 copies for the kernels.
// Forward pass on the tensor cores (the default where nx is a multiple of 8):
//   k_conv_tc      every layer as 27 tcgen05.mma per z plane over shared-memory halo
//                  planes (described below); k_conv_fwd then serves the backward pass and
//                  grids the tensor-core kernel does not take.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "qg_internal.h"
#include "tc_common.cuh"

namespace {

constexpr int TX = 8, TY = 8, TZ = 4;
constexpr int TV = TX * TY * TZ;  // voxels per tile
constexpr int HX = TX + 2, HY = TY + 2, HZ = TZ + 2;
constexpr int HV = HX * HY * HZ;
constexpr int kLayers = 4;
constexpr int kCin[kLayers] = {2, 16, 16, 16};
constexpr int kCout[kLayers] = {16, 16, 16, 1};

constexpr int wcount(int l) { return kCin[l] * kCout[l] * 27; }
constexpr int lsize(int l) { return wcount(l) + kCout[l]; }
constexpr int woff(int l) { return l == 0 ? 0 : woff(l - 1) + lsize(l - 1); }
constexpr int kParams = woff(kLayers);  // 15169

struct Grid {
    int nx, ny, nz;
    int tx, ty, tz;  // tiles per axis
    long long N;
};

__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

__device__ __forceinline__ float ldf(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ float ldf(const float* p) { return *p; }
__device__ __forceinline__ void stf(__nv_bfloat16* p, float v) { *p = __float2bfloat16(v); }
__device__ __forceinline__ void stf(float* p, float v) { *p = v; }

// out (B x COUT x N) = conv(in (B x CIN x N)); W bf16 [COUT][CIN][27]; bias may be null.
// mask (B x COUT x N, may be null): out *= (mask > 0) (ReLU derivative of the layer below).
template <int CIN, int COUT, bool RELU, typename TI, typename TO>
__global__ void __launch_bounds__(TV) k_conv_fwd(const TI* __restrict__ in, const __nv_bfloat16* __restrict__ W,
                                                 const float* __restrict__ bias, TO* __restrict__ out,
                                                 const __nv_bfloat16* __restrict__ mask, Grid g) {
    __shared__ float tin[HV];
    __shared__ __align__(16) float w[27 * COUT];
    const int tile = blockIdx.x, b = blockIdx.y;
    const int bx = (tile % g.tx) * TX, by = ((tile / g.tx) % g.ty) * TY, bz = (tile / (g.tx * g.ty)) * TZ;
    const int t = threadIdx.x;
    const int lx = t % TX, ly = (t / TX) % TY, lz = t / (TX * TY);
    const int x = bx + lx, y = by + ly, z = bz + lz;
    const bool inside = x < g.nx && y < g.ny && z < g.nz;
    float acc[COUT];
#pragma unroll
    for (int c = 0; c < COUT; ++c) acc[c] = bias ? bias[c] : 0.f;
    const TI* inb = in + (long long)b * CIN * g.N;
    for (int ci = 0; ci < CIN; ++ci) {
        const TI* ic = inb + (long long)ci * g.N;
        for (int i = t; i < HV; i += TV) {
            const int hx = i % HX, hy = (i / HX) % HY, hz = i / (HX * HY);
            const int gx = wrapi(bx + hx - 1, g.nx), gy = wrapi(by + hy - 1, g.ny), gz = wrapi(bz + hz - 1, g.nz);
            tin[i] = ldf(ic + gx + (long long)g.nx * (gy + (long long)g.ny * gz));
        }
        for (int i = t; i < 27 * COUT; i += TV) {
            const int tap = i / COUT, co = i % COUT;
            w[i] = __bfloat162float(W[((long long)co * CIN + ci) * 27 + tap]);
        }
        __syncthreads();
#pragma unroll
        for (int tap = 0; tap < 27; ++tap) {
            const int dx = tap % 3, dy = (tap / 3) % 3, dz = tap / 9;
            const float xv = tin[(lx + dx) + HX * ((ly + dy) + HY * (lz + dz))];
            if constexpr (COUT % 4 == 0) {
#pragma unroll
                for (int c = 0; c < COUT; c += 4) {
                    const float4 wv = *reinterpret_cast<const float4*>(&w[tap * COUT + c]);
                    acc[c] += wv.x * xv;
                    acc[c + 1] += wv.y * xv;
                    acc[c + 2] += wv.z * xv;
                    acc[c + 3] += wv.w * xv;
                }
            } else {
#pragma unroll
                for (int c = 0; c < COUT; ++c) acc[c] += w[tap * COUT + c] * xv;
            }
        }
        __syncthreads();
    }
    if (!inside) return;
    const long long v = x + (long long)g.nx * (y + (long long)g.ny * z);
#pragma unroll
    for (int c = 0; c < COUT; ++c) {
        float o = acc[c];
        if (RELU) o = fmaxf(o, 0.f);
        const long long idx = ((long long)b * COUT + c) * g.N + v;
        if (mask && __bfloat162float(mask[idx]) <= 0.f) o = 0.f;
        stf(out + idx, o);
    }
}

// Partial weight/bias gradients of one tile: part[blk][co][ci*27 + tap] and part[blk][COUT*CIN*27 + co].
// Thread k < CIN*27 handles (ci, tap) for all co; bias by threads k < COUT.
template <int CIN, int COUT, typename TI>
__global__ void __launch_bounds__(448) k_conv_wgrad(const TI* __restrict__ in, const float* __restrict__ dout,
                                                    float* __restrict__ part, Grid g) {
    __shared__ __nv_bfloat16 tin[CIN * HV];  // the layer inputs are bf16 activations
    __shared__ __align__(16) float dt[TV * COUT];  // [voxel][co]
    const int tile = blockIdx.x, b = blockIdx.y;
    const int bx = (tile % g.tx) * TX, by = ((tile / g.tx) % g.ty) * TY, bz = (tile / (g.tx * g.ty)) * TZ;
    const int t = threadIdx.x;
    const TI* inb = in + (long long)b * CIN * g.N;
    for (int i = t; i < CIN * HV; i += blockDim.x) {
        const int ci = i / HV, h = i % HV;
        const int hx = h % HX, hy = (h / HX) % HY, hz = h / (HX * HY);
        const int gx = wrapi(bx + hx - 1, g.nx), gy = wrapi(by + hy - 1, g.ny), gz = wrapi(bz + hz - 1, g.nz);
        tin[i] = __float2bfloat16(ldf(inb + (long long)ci * g.N + gx + (long long)g.nx * (gy + (long long)g.ny * gz)));
    }
    for (int i = t; i < TV * COUT; i += blockDim.x) {
        const int vx = i / COUT, co = i % COUT;
        const int lx = vx % TX, ly = (vx / TX) % TY, lz = vx / (TX * TY);
        const int x = bx + lx, y = by + ly, z = bz + lz;
        float d = 0.f;  // voxels outside the grid (partial tiles) contribute nothing
        if (x < g.nx && y < g.ny && z < g.nz)
            d = dout[((long long)b * COUT + co) * g.N + x + (long long)g.nx * (y + (long long)g.ny * z)];
        dt[i] = d;
    }
    __syncthreads();
    const long long blk = (long long)b * gridDim.x + tile;
    float* pb = part + blk * (COUT * CIN * 27 + COUT);
    if (t < CIN * 27) {
        const int ci = t / 27, tap = t % 27;
        const int dx = tap % 3, dy = (tap / 3) % 3, dz = tap / 9;
        float acc[COUT];
#pragma unroll
        for (int c = 0; c < COUT; ++c) acc[c] = 0.f;
        for (int vx = 0; vx < TV; ++vx) {
            const int lx = vx % TX, ly = (vx / TX) % TY, lz = vx / (TX * TY);
            const float xv = __bfloat162float(tin[ci * HV + (lx + dx) + HX * ((ly + dy) + HY * (lz + dz))]);
            if constexpr (COUT % 4 == 0) {
#pragma unroll
                for (int c = 0; c < COUT; c += 4) {
                    const float4 d4 = *reinterpret_cast<const float4*>(&dt[vx * COUT + c]);
                    acc[c] += d4.x * xv;
                    acc[c + 1] += d4.y * xv;
                    acc[c + 2] += d4.z * xv;
                    acc[c + 3] += d4.w * xv;
                }
            } else {
#pragma unroll
                for (int c = 0; c < COUT; ++c) acc[c] += dt[vx * COUT + c] * xv;
            }
        }
#pragma unroll
        for (int c = 0; c < COUT; ++c) pb[c * CIN * 27 + t] = acc[c];
    }
    if (t < COUT) {
        float s = 0.f;
        for (int vx = 0; vx < TV; ++vx) s += dt[vx * COUT + t];
        pb[COUT * CIN * 27 + t] = s;
    }
}

// grad[i] = sum over blocks of part[blk][i], blocks in order
__global__ void k_reduce_parts(const float* __restrict__ part, int nblk, int n, float* __restrict__ grad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.f;
    for (int k = 0; k < nblk; ++k) s += part[(long long)k * n + i];
    grad[i] = s;
}

// transposed, flipped weights of one layer: Wt[ci][co][26 - tap] = W[co][ci][tap]
__global__ void k_transpose_w(const __nv_bfloat16* __restrict__ W, int cin, int cout, __nv_bfloat16* __restrict__ Wt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cin * cout * 27) return;
    const int co = i / (cin * 27), ci = (i / 27) % cin, tap = i % 27;
    Wt[((long long)ci * cout + co) * 27 + (26 - tap)] = W[i];
}

__global__ void k_to_bf16(const float* __restrict__ src, int n, __nv_bfloat16* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = __float2bfloat16(src[i]);
}

__global__ void k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, int n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// rms[s] = sqrt(mean_i R[s][i]^2) (one block per state)
__global__ void k_rms(const double* __restrict__ R, long long ld, long long N, double* __restrict__ rms) {
    __shared__ double red[32];
    const double* r = R + (long long)blockIdx.x * ld;
    double s = 0.0;
    for (long long i = threadIdx.x; i < N; i += blockDim.x) s += r[i] * r[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        const double v = sqrt(tot / (double)N);
        rms[blockIdx.x] = v > 0.0 ? v : 1.0;
    }
}

// network input of state s: [R[s] / rms[s], V / vscale] as bf16 (B x 2 x N)
__global__ void k_make_input(const double* __restrict__ R, long long ld, const double* __restrict__ V, double vscale,
                             const double* __restrict__ rms, long long N, int B, __nv_bfloat16* __restrict__ in) {
    const long long total = (long long)B * N;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(e / N);
        const long long i = e - (long long)s * N;
        in[((long long)s * 2) * N + i] = __double2bfloat16(R[(long long)s * ld + i] / rms[s]);
        in[((long long)s * 2 + 1) * N + i] = __double2bfloat16(V[i] / vscale);
    }
}

// out[s][i] (+)= rms[s] * p[s][i]
__global__ void k_emit(const float* __restrict__ p, const double* __restrict__ rms, long long N, int B, double* __restrict__ out,
                       long long ldo, int accumulate) {
    const long long total = (long long)B * N;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(e / N);
        const long long i = e - (long long)s * N;
        const double v = rms[s] * (double)p[e];
        double* o = out + (long long)s * ldo + i;
        *o = accumulate ? *o + v : v;
    }
}

// MSE loss terms: dp = 2 (p - y/rms) / sum_s |y_s/rms_s|^2, lossv[e] = (p - t)^2, tnorm[e] = t^2
__global__ void k_loss(const float* __restrict__ p, const double* __restrict__ Y, long long ldy,
                       const double* __restrict__ rms, long long N, int B, float* __restrict__ dp,
                       double* __restrict__ acc2) {
    __shared__ double red[2][32];
    const long long total = (long long)B * N;
    double se = 0.0, st = 0.0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(e / N);
        const long long i = e - (long long)s * N;
        const double tv = Y[(long long)s * ldy + i] / rms[s];
        const double d = (double)p[e] - tv;
        dp[e] = (float)(2.0 * d);
        se += d * d;
        st += tv * tv;
    }
    for (int o = 16; o > 0; o >>= 1) {
        se += __shfl_xor_sync(0xffffffffu, se, o);
        st += __shfl_xor_sync(0xffffffffu, st, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = se;
        red[1][threadIdx.x >> 5] = st;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, bsum = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a += red[0][w];
            bsum += red[1][w];
        }
        acc2[2 * blockIdx.x] = a;
        acc2[2 * blockIdx.x + 1] = bsum;
    }
}

__global__ void k_scale_f(float* __restrict__ x, long long n, const double* __restrict__ inv) {
    const float s = (float)inv[0];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] *= s;
}


// ---------------------------------------------------------------------------
// The network layers on the 5th-generation tensor cores (sm_100a).
// One CTA (4 warps) owns a column block of CX x CY voxels of one state (two groups of 8
// x-voxels, each one M = 128 MMA with its own 16-column accumulator) and marches CZ
// planes in z. The input's halo planes (CX+2 x CY+2 voxels) sit in shared memory split
// into two 8-channel halves, each voxel's 8 channels one 16-byte row, so that operand A
// of one tap -- 128 voxels (x fastest) x 16 input channels -- is the canonical K-major
// layout without swizzle at a shifted start address: each run of 8 voxels along x is one
// core matrix (8 rows of 16 bytes), consecutive y rows are HXC * 16 bytes apart (SBO)
// and the second channel half one half-plane further (LBO). The 27 taps are then 27
// tcgen05.mma.kind::f16 (M 128, N 16, K 16, BF16 in, FP32 accumulator in TMEM) with no
// im2col copy; the weights sit as [tap][channel half][co][8 ci] (LBO 256 B, SBO 128 B).
// After the MMAs of plane z are committed the CTA loads halo plane z + 2 (ring of 4),
// then reads the accumulator back with tcgen05.ld (one TMEM lane per voxel), adds the
// bias, applies ReLU where the layer has one and stores (BF16 activations, FP32 for the
// last layer). Layers with fewer channels use the same 16 x 16 MMA: the missing input
// channels are zero in the halo, the missing outputs have zero weights and are not
// stored. Same periodic convolution as k_conv_fwd; the products are summed in a
// different order (per tap on the tensor cores).
using namespace qg::tc;

constexpr int CX = 16, CY = 16, CZ = 8;         // voxels of a CTA's column block; z planes per CTA
constexpr int kGroupsX = CX / 8;                // M = 128 groups (8 x-voxels x 16 y rows) per plane
constexpr int HXC = CX + 2, HYC = CY + 2;
constexpr int kHalfB = HXC * HYC * 16;          // one 8-channel half of a halo plane (5184 B)
constexpr int kSlotB = 2 * kHalfB;              // one halo plane
constexpr int kSlots = 4;
constexpr int kWB = 27 * 512;                   // weights, bf16 [tap][half][co][8]
// shared memory: the halo ring, the weights, the mbarrier and the TMEM address (54 KB;
// a tap's operand reaches at most the end of the ring)
constexpr int kConvTcSmem = kSlots * kSlotB + kWB + 64;
constexpr uint32_t kIdescConv = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint64_t desc_nosw(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFF) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_conv(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdescConv), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ int wrap_any(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// out (B x COUT x N) = act(conv(in (B x CIN x N)) + bias); W bf16 [COUT][CIN][27];
// CIN, COUT <= 16 (the MMA is always 16 x 16 per tap: missing input channels are zero
// in the halo, missing output channels have zero weights and are not stored). Grid:
// x = (x block, y block, z slab), y = state. Requires nx % 8 == 0; in a last x block of
// 8 voxels the second group computes on periodic copies and stores nothing.
template <int CIN, int COUT, bool RELU, typename TO>
__global__ void __launch_bounds__(128) k_conv_tc(const __nv_bfloat16* __restrict__ in,
                                                 const __nv_bfloat16* __restrict__ W,
                                                 const float* __restrict__ bias, TO* __restrict__ out,
                                                 Grid g, int tiles_y, int* err) {
    static_assert(CIN >= 1 && CIN <= 16 && COUT >= 1 && COUT <= 16, "16 x 16 channel MMA");
    extern __shared__ __align__(128) unsigned char csm[];
    unsigned char* halo = csm;
    unsigned char* wsm = csm + kSlots * kSlotB;
    uint64_t* bar = reinterpret_cast<uint64_t*>(wsm + kWB);
    volatile uint32_t* tslot = reinterpret_cast<volatile uint32_t*>(bar + 1);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int txb = (g.nx + CX - 1) / CX;
    int blk = blockIdx.x;
    const int xb = blk % txb;
    blk /= txb;
    const int yb = blk % tiles_y;
    const int zs = blk / tiles_y;
    const int b = blockIdx.y;
    const int x0 = xb * CX, y0 = yb * CY, z0 = zs * CZ, z1 = min(g.nz, z0 + CZ);

    if (t == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32((const void*)tslot)),
                     "r"(32)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // weights: element ((tap * 2 + h) * 16 + co) * 8 + j = W[co][h * 8 + j][tap] (zero past CIN, COUT)
    __nv_bfloat16* wb = reinterpret_cast<__nv_bfloat16*>(wsm);
    for (int i = t; i < 27 * 256; i += 128) {
        const int j = i & 7, co = (i >> 3) & 15, h = (i >> 7) & 1, tap = i >> 8, ci = h * 8 + j;
        wb[i] = (ci < CIN && co < COUT) ? W[(co * CIN + ci) * 27 + tap] : __float2bfloat16(0.f);
    }
    if constexpr (CIN < 16) {
        // the channels the input lacks stay zero in every halo plane
        for (int i = t; i < kSlots * kSlotB / 16; i += 128) reinterpret_cast<uint4*>(halo)[i] = make_uint4(0, 0, 0, 0);
        __syncthreads();
    }
    const __nv_bfloat16* inb = in + (long long)b * CIN * g.N;
    const int xl0 = wrap_any(x0 - 1, g.nx), xr0 = wrap_any(x0 + CX, g.nx);
    int xm[kGroupsX];  // start of each 8-voxel interior run (periodic past nx; multiples of 8)
#pragma unroll
    for (int q = 0; q < kGroupsX; ++q) xm[q] = wrap_any(x0 + 8 * q, g.nx);
    auto load_plane = [&](int z) {  // z in [-1, nz]: halo plane z into slot (z + 4) % 4
        const int zz = wrap_any(z, g.nz);
        unsigned char* dst = halo + ((z + 4) & 3) * kSlotB;
        // one (channel, y row) per step: each run of 8 interior voxels as one 16-byte load
        // (x0 and nx are multiples of 8), the two periodic edge voxels as single loads
        for (int e = t; e < CIN * HYC; e += 128) {
            // channels on consecutive lanes: 8 lanes fill one voxel's 16-byte row
            const int ci = e % CIN, yh = e / CIN;
            const long long row = (long long)ci * g.N + (long long)g.nx * (wrap_any(y0 + yh - 1, g.ny) + (long long)g.ny * zz);
            __nv_bfloat16 vals[HXC];
            vals[0] = inb[row + xl0];
            vals[HXC - 1] = inb[row + xr0];
#pragma unroll
            for (int q = 0; q < kGroupsX; ++q) {
                const uint4 mid = *reinterpret_cast<const uint4*>(inb + row + xm[q]);
                const __nv_bfloat16* mv = reinterpret_cast<const __nv_bfloat16*>(&mid);
#pragma unroll
                for (int i = 0; i < 8; ++i) vals[1 + 8 * q + i] = mv[i];
            }
            __nv_bfloat16* rowdst = reinterpret_cast<__nv_bfloat16*>(dst + (ci >> 3) * kHalfB + yh * HXC * 16) + (ci & 7);
#pragma unroll
            for (int xh = 0; xh < HXC; ++xh) rowdst[xh * 8] = vals[xh];
        }
    };
    load_plane(z0 - 1);
    load_plane(z0);
    load_plane(z0 + 1);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // thread stores -> tensor core reads
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t hbase = smem_u32(halo), wbase = smem_u32(wsm);
    float bs[COUT];
#pragma unroll
    for (int c = 0; c < COUT; ++c) bs[c] = bias[c];
    const int m = warp * 32 + lane, xl = m & 7, yl = m >> 3;
    uint32_t phase = 0;
    bool bad = false;
    for (int z = z0; z < z1; ++z) {
        if (t == 0) {
#pragma unroll 1
            for (int tap = 0; tap < 27; ++tap) {
                const int dx = tap % 3, dy = (tap / 3) % 3, dz = tap / 9;
                const uint64_t bd = desc_nosw(wbase + tap * 512, 256, 128);
#pragma unroll
                for (int q = 0; q < kGroupsX; ++q) {
                    const uint32_t a =
                        hbase + (uint32_t)((((z - 1 + dz) + 4) & 3) * kSlotB + (dy * HXC + dx + 8 * q) * 16);
                    umma_conv(tmem + (uint32_t)(16 * q), desc_nosw(a, kHalfB, HXC * 16), bd, tap ? 1u : 0u);
                }
            }
            umma_commit(bar);
        }
        if (z + 1 < z1) load_plane(z + 2);  // for plane z + 1 (the slot of plane z - 2, not read now)
        const bool ok = mbar_wait(bar, phase);
        if (__syncthreads_or(!ok)) {
            bad = true;
            break;
        }
        phase ^= 1u;
        tc_fence_after();
        const int y = y0 + yl;
#pragma unroll
        for (int q = 0; q < kGroupsX; ++q) {
            uint32_t r[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(16 * q), r);
            tmem_wait_ld();
            const int x = x0 + 8 * q + xl;
            if (y < g.ny && x < g.nx) {
                const long long v = x + (long long)g.nx * (y + (long long)g.ny * z);
                TO* ob = out + (long long)b * COUT * g.N + v;
#pragma unroll
                for (int c = 0; c < COUT; ++c) {
                    float o = __uint_as_float(r[c]) + bs[c];
                    if (RELU) o = fmaxf(o, 0.f);
                    stf(ob + (long long)c * g.N, o);
                }
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    if (bad) {
        if (t == 0) {
            atomicExch(err, (int)QG_ERR_TIMEOUT);
            mbar_wait(bar, phase);  // bounded: the MMAs in flight finish before TMEM is freed
        }
        __syncthreads();
    }
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32) : "memory");
    }
}

bool conv_tc_ok(const Grid& g, int B) {
    if (g.nx % 8 != 0 || B > 65535) return false;
    const long long nblk = (long long)((g.nx + CX - 1) / CX) * ((g.ny + CY - 1) / CY) * ((g.nz + CZ - 1) / CZ);
    return nblk <= 0x7fffffffLL;
}

template <int CIN, int COUT, bool RELU, typename TO>
int launch_conv_tc(const __nv_bfloat16* in, const __nv_bfloat16* W, const float* bias, TO* out, const Grid& g, int B,
                   int* err, cudaStream_t st) {
    const int tiles_y = (g.ny + CY - 1) / CY;
    const long long nblk = (long long)((g.nx + CX - 1) / CX) * tiles_y * ((g.nz + CZ - 1) / CZ);
    QG_CUDA_TRY(cudaFuncSetAttribute(k_conv_tc<CIN, COUT, RELU, TO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kConvTcSmem));
    k_conv_tc<CIN, COUT, RELU, TO><<<dim3((unsigned)nblk, B), 128, kConvTcSmem, st>>>(in, W, bias, out, g, tiles_y, err);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}
}  // namespace

struct qg_learned_s {
    qg_context ctx = nullptr;
    DevBuf master, adam_m, adam_v, grad, wbf, wtbf;  // params FP32 / BF16, transposed BF16 weights
    DevBuf act, dact, part, small, loss_acc;         // activations, gradients, partials, scratch
    int step = 0;
    bool tensor_cores = true;  // the forward layers on tcgen05 where the grid allows
};

namespace {

Grid make_grid(int nx, int ny, int nz) {
    Grid g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.tx = (nx + TX - 1) / TX; g.ty = (ny + TY - 1) / TY; g.tz = (nz + TZ - 1) / TZ;
    g.N = (long long)nx * ny * nz;
    return g;
}

// forward through the 4 layers; keeps every layer's output in L->act:
//   act = [in (B x 2 x N) | h1 | h2 | h3 (B x 16 x N each), bf16] and p (B x N, float) after them
int forward(qg_learned L, const Grid& g, int B, cudaStream_t st, __nv_bfloat16** acts, float** pout) {
    const size_t N = (size_t)g.N;
    const size_t need = (size_t)B * N * (2 + 16 * 3) * sizeof(__nv_bfloat16) + (size_t)B * N * sizeof(float) + 256;
    QG_TRY(L->act.reserve(need));
    __nv_bfloat16* a0 = L->act.as<__nv_bfloat16>();
    __nv_bfloat16* a1 = a0 + (size_t)B * 2 * N;
    __nv_bfloat16* a2 = a1 + (size_t)B * 16 * N;
    __nv_bfloat16* a3 = a2 + (size_t)B * 16 * N;
    float* p = reinterpret_cast<float*>(a3 + (size_t)B * 16 * N);
    acts[0] = a0; acts[1] = a1; acts[2] = a2; acts[3] = a3;
    *pout = p;
    const __nv_bfloat16* W = L->wbf.as<__nv_bfloat16>();
    const float* P = L->master.as<float>();  // biases are read in FP32
    if (L->tensor_cores && conv_tc_ok(g, B)) {
        // every layer on tcgen05 (16 x 16 channel MMAs; layer 1 pads its 2 input channels,
        // layer 4 its 1 output channel)
        int* err = L->ctx->dev_status;
        QG_TRY((launch_conv_tc<2, 16, true>(a0, W + woff(0), P + woff(0) + wcount(0), a1, g, B, err, st)));
        QG_TRY((launch_conv_tc<16, 16, true>(a1, W + woff(1), P + woff(1) + wcount(1), a2, g, B, err, st)));
        QG_TRY((launch_conv_tc<16, 16, true>(a2, W + woff(2), P + woff(2) + wcount(2), a3, g, B, err, st)));
        QG_TRY((launch_conv_tc<16, 1, false>(a3, W + woff(3), P + woff(3) + wcount(3), p, g, B, err, st)));
        return QG_OK;
    }
    const dim3 grid(g.tx * g.ty * g.tz, B);
    k_conv_fwd<2, 16, true, __nv_bfloat16, __nv_bfloat16><<<grid, TV, 0, st>>>(a0, W + woff(0), P + woff(0) + wcount(0), a1, nullptr, g);
    k_conv_fwd<16, 16, true, __nv_bfloat16, __nv_bfloat16><<<grid, TV, 0, st>>>(a1, W + woff(1), P + woff(1) + wcount(1), a2, nullptr, g);
    k_conv_fwd<16, 16, true, __nv_bfloat16, __nv_bfloat16><<<grid, TV, 0, st>>>(a2, W + woff(2), P + woff(2) + wcount(2), a3, nullptr, g);
    k_conv_fwd<16, 1, false, __nv_bfloat16, float><<<grid, TV, 0, st>>>(a3, W + woff(3), P + woff(3) + wcount(3), p, nullptr, g);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

int prepare_input(qg_learned L, const Grid& g, int B, const double* R, long long ldr, const double* V,
                  double vscale, cudaStream_t st, double** rms_out) {
    QG_TRY(L->small.reserve((size_t)(B + 8) * sizeof(double)));
    double* rms = L->small.as<double>();
    k_rms<<<B, 256, 0, st>>>(R, ldr, g.N, rms);
    const size_t N = (size_t)g.N;
    const size_t need = (size_t)B * N * (2 + 16 * 3) * sizeof(__nv_bfloat16) + (size_t)B * N * sizeof(float) + 256;
    QG_TRY(L->act.reserve(need));
    k_make_input<<<148 * 8, 256, 0, st>>>(R, ldr, V, vscale, rms, g.N, B, L->act.as<__nv_bfloat16>());
    QG_CUDA_TRY(cudaGetLastError());
    *rms_out = rms;
    return QG_OK;
}

int refresh_weights(qg_learned L, cudaStream_t st) {
    k_to_bf16<<<(kParams + 255) / 256, 256, 0, st>>>(L->master.as<float>(), kParams, L->wbf.as<__nv_bfloat16>());
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

// loss and parameter gradient (L->grad) of one batch; leaves the loss on the host
int loss_and_grad(qg_learned L, const Grid& g, int B, const double* R, long long ldr, const double* V, double vscale,
                  const double* Y, long long ldy, cudaStream_t st, double* loss) {
    double* rms = nullptr;
    QG_TRY(prepare_input(L, g, B, R, ldr, V, vscale, st, &rms));
    __nv_bfloat16* a[4];
    float* p = nullptr;
    QG_TRY(forward(L, g, B, st, a, &p));
    const size_t N = (size_t)g.N;
    // gradient buffers: dp (B x N) and two B x 16 x N float buffers
    QG_TRY(L->dact.reserve((size_t)B * N * (1 + 32) * sizeof(float)));
    float* dp = L->dact.as<float>();
    float* dA = dp + (size_t)B * N;
    float* dB = dA + (size_t)B * 16 * N;
    const int nlb = 148 * 4;
    QG_TRY(L->loss_acc.reserve((size_t)(2 * nlb + 4) * sizeof(double)));
    double* acc2 = L->loss_acc.as<double>();
    k_loss<<<nlb, 256, 0, st>>>(p, Y, ldy, rms, g.N, B, dp, acc2);
    std::vector<double> h(2 * nlb);
    QG_CUDA_TRY(cudaMemcpyAsync(h.data(), acc2, 2 * nlb * sizeof(double), cudaMemcpyDeviceToHost, st));
    QG_CUDA_TRY(cudaStreamSynchronize(st));
    double se = 0.0, stt = 0.0;
    for (int i = 0; i < nlb; ++i) {
        se += h[2 * i];
        stt += h[2 * i + 1];
    }
    const double inv = stt > 0.0 ? 1.0 / stt : 1.0;
    *loss = se * inv;
    // dp <- dp / sum |t|^2
    QG_CUDA_TRY(cudaMemcpyAsync(acc2 + 2 * nlb, &inv, sizeof(double), cudaMemcpyHostToDevice, st));
    k_scale_f<<<148 * 8, 256, 0, st>>>(dp, (long long)B * g.N, acc2 + 2 * nlb);

    const dim3 grid(g.tx * g.ty * g.tz, B);
    const int nblk = grid.x * grid.y;
    const int maxl = 16 * 16 * 27 + 16;
    QG_TRY(L->part.reserve((size_t)nblk * maxl * sizeof(float)));
    float* part = L->part.as<float>();
    float* G = L->grad.as<float>();
    const __nv_bfloat16* Wt = L->wtbf.as<__nv_bfloat16>();
    const __nv_bfloat16* W = L->wbf.as<__nv_bfloat16>();
    for (int l = 0; l < kLayers; ++l)
        k_transpose_w<<<(wcount(l) + 255) / 256, 256, 0, st>>>(W + woff(l), kCin[l], kCout[l],
                                                                L->wtbf.as<__nv_bfloat16>() + woff(l));
    // layer 4 (16 -> 1, linear)
    k_conv_wgrad<16, 1, __nv_bfloat16><<<grid, 448, 0, st>>>(a[3], dp, part, g);
    k_reduce_parts<<<(lsize(3) + 255) / 256, 256, 0, st>>>(part, nblk, lsize(3), G + woff(3));
    k_conv_fwd<1, 16, false, float, float><<<grid, TV, 0, st>>>(dp, Wt + woff(3), nullptr, dA, a[3], g);
    // layer 3 (16 -> 16)
    k_conv_wgrad<16, 16, __nv_bfloat16><<<grid, 448, 0, st>>>(a[2], dA, part, g);
    k_reduce_parts<<<(lsize(2) + 255) / 256, 256, 0, st>>>(part, nblk, lsize(2), G + woff(2));
    k_conv_fwd<16, 16, false, float, float><<<grid, TV, 0, st>>>(dA, Wt + woff(2), nullptr, dB, a[2], g);
    // layer 2 (16 -> 16)
    k_conv_wgrad<16, 16, __nv_bfloat16><<<grid, 448, 0, st>>>(a[1], dB, part, g);
    k_reduce_parts<<<(lsize(1) + 255) / 256, 256, 0, st>>>(part, nblk, lsize(1), G + woff(1));
    k_conv_fwd<16, 16, false, float, float><<<grid, TV, 0, st>>>(dB, Wt + woff(1), nullptr, dA, a[1], g);
    // layer 1 (2 -> 16)
    k_conv_wgrad<2, 16, __nv_bfloat16><<<grid, 448, 0, st>>>(a[0], dA, part, g);
    k_reduce_parts<<<(lsize(0) + 255) / 256, 256, 0, st>>>(part, nblk, lsize(0), G + woff(0));
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

}  // namespace

extern "C" {

int qg_learned_num_params(void) { return kParams; }

int qg_hamiltonian_set_learned(qg_hamiltonian h, qg_learned nn, double vscale) {
    if (!h || (nn && (nn->ctx != h->ctx || !(vscale > 0)))) return QG_ERR_INVALID;
    h->learned = nn;
    h->learned_vscale = nn ? vscale : 1.0;
    return QG_OK;
}

int qg_learned_create(qg_context ctx, qg_learned* out) {
    if (!ctx || !out) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(ctx->device));
    qg_learned L = new qg_learned_s();
    L->ctx = ctx;
    const size_t pb = (size_t)kParams * sizeof(float);
    int rc = L->master.reserve(pb);
    if (rc == QG_OK) rc = L->adam_m.reserve(pb);
    if (rc == QG_OK) rc = L->adam_v.reserve(pb);
    if (rc == QG_OK) rc = L->grad.reserve(pb);
    if (rc == QG_OK) rc = L->wbf.reserve((size_t)kParams * sizeof(__nv_bfloat16));
    if (rc == QG_OK) rc = L->wtbf.reserve((size_t)kParams * sizeof(__nv_bfloat16));
    if (rc != QG_OK) {
        delete L;
        return rc;
    }
    cudaMemsetAsync(L->master.ptr, 0, pb, ctx->stream);
    cudaMemsetAsync(L->adam_m.ptr, 0, pb, ctx->stream);
    cudaMemsetAsync(L->adam_v.ptr, 0, pb, ctx->stream);
    refresh_weights(L, ctx->stream);
    ctx->live_hamiltonians++;
    *out = L;
    return QG_OK;
}

int qg_learned_destroy(qg_learned L) {
    if (!L) return QG_ERR_INVALID;
    cudaSetDevice(L->ctx->device);
    cudaStreamSynchronize(L->ctx->stream);
    for (DevBuf* b : {&L->master, &L->adam_m, &L->adam_v, &L->grad, &L->wbf, &L->wtbf, &L->act, &L->dact, &L->part,
                      &L->small, &L->loss_acc})
        b->release();
    L->ctx->live_hamiltonians--;
    delete L;
    return QG_OK;
}

int qg_learned_set_params(qg_learned L, const float* params, int n) {
    if (!L || !params || n != kParams) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(L->ctx->device));
    QG_CUDA_TRY(cudaMemcpyAsync(L->master.ptr, params, (size_t)n * sizeof(float), cudaMemcpyHostToDevice,
                                L->ctx->stream));
    QG_TRY(refresh_weights(L, L->ctx->stream));
    QG_CUDA_TRY(cudaStreamSynchronize(L->ctx->stream));
    return QG_OK;
}

int qg_learned_get_params(qg_learned L, float* params, int n) {
    if (!L || !params || n != kParams) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(L->ctx->device));
    QG_CUDA_TRY(cudaMemcpyAsync(params, L->master.ptr, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost,
                                L->ctx->stream));
    QG_CUDA_TRY(cudaStreamSynchronize(L->ctx->stream));
    return QG_OK;
}

int qg_learned_set_tensor_cores(qg_learned L, int on) {
    if (!L) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaStreamSynchronize(L->ctx->stream));
    L->tensor_cores = on != 0;
    return QG_OK;
}

int qg_learned_apply_d(qg_learned L, int nx, int ny, int nz, int ns, const double* R, long long ldr, const double* V,
                       double vscale, double* out, long long ldo, int accumulate) {
    if (!L || nx < 3 || ny < 3 || nz < 3 || ns <= 0 || !R || !V || !out || !(vscale > 0)) return QG_ERR_INVALID;
    const Grid g = make_grid(nx, ny, nz);
    if (ldr < g.N || ldo < g.N || ns > 65535) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(L->ctx->device));
    cudaStream_t st = L->ctx->stream;
    // states in chunks whose activations (50 bf16 channels + the float output per
    // voxel) stay within about 4 GB
    const long long per_state = g.N * (50 * 2 + 4);
    const int chunk = (int)std::max<long long>(1, std::min<long long>(ns, (4LL << 30) / per_state));
    for (int s0 = 0; s0 < ns; s0 += chunk) {
        const int B = std::min(chunk, ns - s0);
        double* rms = nullptr;
        QG_TRY(prepare_input(L, g, B, R + (long long)s0 * ldr, ldr, V, vscale, st, &rms));
        __nv_bfloat16* a[4];
        float* p = nullptr;
        QG_TRY(forward(L, g, B, st, a, &p));
        k_emit<<<148 * 8, 256, 0, st>>>(p, rms, g.N, B, out + (long long)s0 * ldo, ldo, accumulate);
    }
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

int qg_learned_gradient(qg_learned L, int nx, int ny, int nz, int ns, const double* R, long long ldr, const double* V,
                        double vscale, const double* Y, long long ldy, double* loss, float* grad_host) {
    if (!L || nx < 3 || ny < 3 || nz < 3 || ns <= 0 || !R || !V || !Y || !loss || !(vscale > 0))
        return QG_ERR_INVALID;
    const Grid g = make_grid(nx, ny, nz);
    if (ldr < g.N || ldy < g.N || ns > 65535) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(L->ctx->device));
    QG_TRY(loss_and_grad(L, g, ns, R, ldr, V, vscale, Y, ldy, L->ctx->stream, loss));
    if (grad_host) {
        QG_CUDA_TRY(cudaMemcpyAsync(grad_host, L->grad.ptr, (size_t)kParams * sizeof(float), cudaMemcpyDeviceToHost,
                                    L->ctx->stream));
        QG_CUDA_TRY(cudaStreamSynchronize(L->ctx->stream));
    }
    return QG_OK;
}

int qg_learned_train_step(qg_learned L, int nx, int ny, int nz, int ns, const double* R, long long ldr,
                          const double* V, double vscale, const double* Y, long long ldy, float lr, double* loss) {
    QG_TRY(qg_learned_gradient(L, nx, ny, nz, ns, R, ldr, V, vscale, Y, ldy, loss, nullptr));
    cudaStream_t st = L->ctx->stream;
    L->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)L->step), c2 = 1.f - powf(b2, (float)L->step);
    k_adam<<<(kParams + 255) / 256, 256, 0, st>>>(L->master.as<float>(), L->adam_m.as<float>(), L->adam_v.as<float>(),
                                                  L->grad.as<float>(), kParams, lr, b1, b2, 1e-8f, c1, c2);
    QG_TRY(refresh_weights(L, st));
    return QG_OK;
}

}  // extern "C"
