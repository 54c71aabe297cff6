// FP64-accurate Gram products on the 5th-generation tensor cores' int8 path (sm_100a):
//   C = alpha * A^T B,  A: N x ma, B: N x nc FP64 blocks (column-major, ld N).
// Column j of each block is scaled by 2^-E_j (E_j: the smallest power of two that puts
// its largest value below 127/128) and cut into kI8Slices exact signed slices,
//   a_kj = 2^E_j * sum_t d_t(k, j) 2^-7(t+1),   d_t = rint(128 v_t), v_{t+1} = 128 v_t - d_t,
// |d_0| <= 127, |d_t| <= 64 for t > 0 (the remainder after 7 slices is below 2^-49 of the
// column's largest value). Then
//   C_ij = 2^(Ea_i + Eb_j) * sum_{d=0..6} 2^-7(d+2) * sum_{t+u=d} sum_k a_t(k,i) b_u(k,j),
// the inner sums exact in int32 (tcgen05.mma.cta_group::1.kind::i8), the 7 scale groups
// added in FP64: an FP64-accurate product from 28 int8 products.
//
// Persistent kernel, one CTA per SM, 10 warps:
//   warp 0      TMA producer: for each 64-row K block, the 7 slices of A's 128 rows and of
//               B's 64 rows (64-byte rows, 64-byte swizzle) into one of 2 ring stages (84 KB);
//   warp 1      owns 512 TMEM columns (7 int32 accumulators of 128 x 64, one per scale
//               group); one lane issues the 56 MMAs (M = 128, N = 64, K = 32) of a K block
//               and frees the stage with tcgen05.commit;
//   warps 2-9   epilogue: at the end of a work unit (a tile and a K segment of at most 256
//               blocks, so the int32 sums stay below 7 * 16384 * 127^2 < 2^31) tcgen05.ld of
//               the 7 accumulators, scaled and added in FP64, one partial tile per unit.
// Work units are K-segment-major; k_gram_i8_reduce adds the segments of each tile in a
// fixed order and applies the column scales (deterministic). Every mbarrier wait is
// bounded; on timeout the kernel records QG_ERR_TIMEOUT, all roles stop, the MMAs issued
// are waited for and TMEM is released.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "gram_i8.h"
#include "tc_common.cuh"

namespace qg {
namespace {

using namespace tc;
using tchost::EncodeTiledFn;
using tchost::encode_fn;

constexpr int S = kI8Slices;
constexpr int BM = 128, BN = 64, BK = 64;
constexpr int kThreads = 320;
constexpr int kEpiWarps = 8;
constexpr int kTileA = BM * BK;       // bytes of one A slice tile (8 KB)
constexpr int kTileB = BN * BK;       // bytes of one B slice tile (4 KB)
constexpr int kStageBytes = S * (kTileA + kTileB);
constexpr int kStages = 2;
constexpr int kSegMax = 256;          // K blocks per work unit (int32 bound)
constexpr int kTmemCols = 512;

struct TMapsI8 {
    CUtensorMap a[S];
    CUtensorMap b[S];
};

struct UnitsI8 {
    int tiles_m, tiles_n, ntiles, lower;
    int nseg, kblocks, kb_per_seg, units;
    int ma, nc, ma_split, mb_split, boff;  // A rows of C, B columns used, the slots' split widths, first B column
};

// Column tiles of row tile r: all, or for the lower triangle those the 128 x 64 block
// reaches (j <= i somewhere in it: tj <= 2 r + 1).
__host__ __device__ __forceinline__ int row_tiles(const UnitsI8& u, int r) {
    return u.lower ? min(2 * r + 2, u.tiles_n) : u.tiles_n;
}

__device__ __forceinline__ void tile_coords(int t, const UnitsI8& u, int& ti, int& tj) {
    if (!u.lower) {
        ti = t / u.tiles_n;
        tj = t - ti * u.tiles_n;
        return;
    }
    int r = 0;
    while (r < u.tiles_m - 1 && t >= row_tiles(u, r)) {
        t -= row_tiles(u, r);
        ++r;
    }
    ti = r;
    tj = t;
}

// Shared-memory matrix descriptor of a K-major tile of 64-byte rows written by TMA with
// the 64-byte swizzle: 8-row core groups 512 bytes apart (SBO), descriptor version 1,
// layout type 4 (SWIZZLE_64B); a K step of 32 int8 advances the start address by 32 bytes.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFF) >> 4) | (1ull << 16) | (32ull << 32) | (1ull << 46) | (4ull << 61);
}

// Instruction descriptor, kind::i8: S32 accumulator, signed 8-bit A and B, both K-major,
// N = 64 (n_dim = N >> 3 at bit 17), M = 128 (m_dim = M >> 4 at bit 24).
constexpr uint32_t kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void umma_i8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdescI8), "r"(accumulate)
        : "memory");
}

__global__ void __launch_bounds__(kThreads, 1)
    k_gram_i8(const __grid_constant__ TMapsI8 tm, const UnitsI8 u, double* __restrict__ part, int* err) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(base);
    uint64_t* empty = full + kStages;
    uint64_t* accfull = empty + kStages;
    uint64_t* accempty = accfull + 1;
    uint64_t* done = accempty + 1;
    volatile uint32_t* tmem_slot = reinterpret_cast<volatile uint32_t*>(done + 1);
    volatile int* ctl = reinterpret_cast<volatile int*>(tmem_slot + 1);
    unsigned char* tiles = base + 1024;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < kStages; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(accfull, 1);
        mbar_init(accempty, kEpiWarps);
        mbar_init(done, 1);
        ctl[0] = 0;
        ctl[1] = -1;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32((const void*)tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            int pos = 0;
            for (int unit = blockIdx.x; unit < u.units && !ctl[0]; unit += gridDim.x) {
                const int seg = unit / u.ntiles;
                int ti, tj;
                tile_coords(unit - seg * u.ntiles, u, ti, tj);
                const int kb0 = seg * u.kb_per_seg, kb1 = min(u.kblocks, kb0 + u.kb_per_seg);
                for (int kb = kb0; kb < kb1; ++kb, ++pos) {
                    const int j = pos % kStages, k = pos / kStages;
                    if (k > 0 && !mbar_wait(&empty[j], (uint32_t)(k - 1) & 1u)) {
                        ctl[0] = 1;
                        atomicExch(err, (int)QG_ERR_TIMEOUT);
                        break;
                    }
                    if (ctl[0]) break;
                    unsigned char* st = tiles + (size_t)j * kStageBytes;
                    mbar_expect_tx(&full[j], kStageBytes);
                    const int ya = kb * u.ma_split + ti * BM;
                    const int yb = kb * u.mb_split + u.boff + tj * BN;
#pragma unroll
                    for (int p = 0; p < S; ++p) {
                        tma_load_2d(st + p * kTileA, &tm.a[p], 0, ya, &full[j]);
                        tma_load_2d(st + S * kTileA + p * kTileB, &tm.b[p], 0, yb, &full[j]);
                    }
                    ctl[1] = pos;
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int pos = 0, nunit = 0;
            for (int unit = blockIdx.x; unit < u.units && !ctl[0]; unit += gridDim.x, ++nunit) {
                const int seg = unit / u.ntiles;
                const int kb0 = seg * u.kb_per_seg, kb1 = min(u.kblocks, kb0 + u.kb_per_seg);
                // the accumulators are free once the epilogue has read the last unit's
                if (nunit > 0 && !mbar_wait(accempty, (uint32_t)(nunit - 1) & 1u)) {
                    ctl[0] = 1;
                    atomicExch(err, (int)QG_ERR_TIMEOUT);
                    break;
                }
                bool ok = true;
                for (int kb = kb0; kb < kb1; ++kb, ++pos) {
                    const int j = pos % kStages, k = pos / kStages;
                    ok = mbar_wait(&full[j], (uint32_t)k & 1u);
                    if (!ok || ctl[0]) break;
                    tc_fence_after();
                    const uint32_t st = smem_u32(tiles + (size_t)j * kStageBytes);
                    const bool first = kb == kb0;
#pragma unroll
                    for (int d = 0; d < S; ++d) {
                        const uint32_t dt = tmem + (uint32_t)(d * BN);
#pragma unroll
                        for (int t = 0; t <= d; ++t) {
#pragma unroll
                            for (int kk = 0; kk < BK / 32; ++kk) {
                                const uint64_t ad = sw64_desc(st + t * kTileA) + 2 * kk;
                                const uint64_t bd = sw64_desc(st + S * kTileA + (d - t) * kTileB) + 2 * kk;
                                umma_i8(dt, ad, bd, (!first || t || kk) ? 1u : 0u);
                            }
                        }
                    }
                    umma_commit(&empty[j]);  // the stage is free once these MMAs have read it
                }
                if (!ok || ctl[0]) {
                    ctl[0] = 1;
                    if (!ok) atomicExch(err, (int)QG_ERR_TIMEOUT);
                    break;
                }
                umma_commit(accfull);  // the accumulators hold this unit
            }
            umma_commit(done);  // completes once every MMA issued above has finished
            mbar_wait(done, 0);
        }
    } else {
        // ---------------- epilogue: TMEM (int32) -> FP64, one partial tile per unit ----------------
        const int lg = warp & 3;            // TMEM lane group this warp may read
        const int half = (warp - 2) >> 2;   // column half (32 of the 64 columns)
        const int row = lg * 32 + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(lg * 32) << 16) + (uint32_t)(half * 32);
        int nunit = 0;
        bool bad = false;
        for (int unit = blockIdx.x; unit < u.units && !bad; unit += gridDim.x, ++nunit) {
            const bool ok = mbar_wait(accfull, (uint32_t)nunit & 1u);
            if (__any_sync(0xffffffffu, !ok || ctl[0] != 0)) {
                bad = true;
                break;
            }
            tc_fence_after();
            double acc[32];
#pragma unroll
            for (int i = 0; i < 32; ++i) acc[i] = 0.0;
#pragma unroll
            for (int d = 0; d < S; ++d) {
                uint32_t r[32];
                tmem_ld32(lane_addr + (uint32_t)(d * BN), r);
                tmem_wait_ld();
                const double sc = ldexp(1.0, -7 * (d + 2));
#pragma unroll
                for (int i = 0; i < 32; ++i) acc[i] += sc * (double)(int)r[i];
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(accempty);
            double* dst = part + (size_t)unit * (BM * BN) + (size_t)row * BN + half * 32;
#pragma unroll
            for (int i = 0; i < 32; i += 2) *reinterpret_cast<double2*>(dst + i) = make_double2(acc[i], acc[i + 1]);
        }
        if (bad) {
            ctl[0] = 1;
            if (lane == 0) atomicExch(err, (int)QG_ERR_TIMEOUT);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0 && lane == 0 && ctl[0]) {
        // wind down: wait (bounded) for the tile loads still in flight
        const int last = ctl[1];
        for (int ps = max(0, last - kStages + 1); ps <= last; ++ps)
            mbar_wait(&full[ps % kStages], (uint32_t)(ps / kStages) & 1u);
    }
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                     : "memory");
    }
}

// C(i, j) = alpha * 2^(Ea_i + Eb_(boff + j)) * sum_seg part[seg][tile(i, j)][i % 128][j % 64],
// C column-major (ld ldc); segments added in order.
__global__ void k_gram_i8_reduce(const double* __restrict__ part, UnitsI8 u, const int* __restrict__ ea,
                                 const int* __restrict__ eb, double alpha, double* __restrict__ C, int ldc) {
    const long long total = (long long)u.ntiles * (BM * BN);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
        const int t = (int)(e / (BM * BN));
        const int off = (int)(e - (long long)t * (BM * BN));
        int ti, tj;
        tile_coords(t, u, ti, tj);
        const int i = ti * BM + off / BN, j = tj * BN + off % BN;
        if (i >= u.ma || j >= u.nc) continue;
        double s = 0.0;
        for (int sg = 0; sg < u.nseg; ++sg) s += part[((size_t)sg * u.ntiles + t) * (BM * BN) + off];
        C[i + (long long)j * ldc] = alpha * ldexp(s, ea[i] + eb[u.boff + j]);
    }
}

// E_j for every column: the exponent of the smallest power of two above max|A_j| * 128/127
// (0 for a zero column).
__global__ void k_col_expo(const double* __restrict__ A, long long N, int m, int* __restrict__ E) {
    __shared__ double red[256];
    for (int j = blockIdx.x; j < m; j += gridDim.x) {
        double mx = 0.0;
        for (long long k = threadIdx.x; k < N; k += blockDim.x) mx = fmax(mx, fabs(A[(long long)j * N + k]));
        red[threadIdx.x] = mx;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            int e = 0;
            if (red[0] > 0.0) frexp(red[0] * (128.0 / 127.0), &e);
            E[j] = e;
        }
        __syncthreads();
    }
}

// The S slices of the N x m block src, K-block-major like the BF16 pieces:
// dst[t][((k / 64) * m + j) * 64 + k % 64] = d_t(k, j), rows N .. kpad-1 zero.
__global__ void k_split_i8(const double* __restrict__ src, long long N, int m, long long kpad,
                           const int* __restrict__ E, int8_t* __restrict__ dst, long long slice_stride) {
    const long long n = kpad * m;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const long long blk = i >> 6;  // (k / 64) * m + j
        const int r = (int)(i & 63);
        const long long kb = blk / m;
        const int j = (int)(blk - kb * m);
        const long long k = kb * BK + r;
        double v = k < N ? ldexp(src[(long long)j * N + k], -E[j]) : 0.0;
#pragma unroll
        for (int t = 0; t < S; ++t) {
            const double d = rint(v * 128.0);
            dst[t * slice_stride + i] = (int8_t)d;
            v = v * 128.0 - d;
        }
    }
}

// Tensor map of one slice: 64-byte rows (one K block of one column), kblocks * m of them; a
// box is `rows` consecutive rows.
int make_map_i8(CUtensorMap* map, const int8_t* ptr, long long kblocks, int m, int rows) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return QG_ERR_UNSUPPORTED;
    const cuuint64_t dims[2] = {(cuuint64_t)BK, (cuuint64_t)(kblocks * m)};
    const cuuint64_t strides[1] = {(cuuint64_t)BK};
    const cuuint32_t box[2] = {BK, (cuuint32_t)rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult rc = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(ptr), dims, strides, box,
                            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return rc == CUDA_SUCCESS ? QG_OK : QG_ERR_UNSUPPORTED;
}

int sm_count_i8() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

int run_i8(I8Gram& g, cudaStream_t st, int ma, int nc, int b_slot, int b_off, bool lower, double alpha, double* C,
           int ldc, int* err) {
    if (ma <= 0 || ma > g.m_slot[0] || nc <= 0 || b_off < 0 || b_off + nc > g.m_slot[b_slot]) return QG_ERR_INVALID;
    TMapsI8 tm;
    std::memset(&tm, 0, sizeof(tm));
    const long long kblocks = g.kpad() / BK;
    const long long ps = g.kpad() * g.mmax;
    const int8_t* A = g.slices[0].as<int8_t>();
    const int8_t* B = g.slices[b_slot].as<int8_t>();
    for (int p = 0; p < S; ++p) {
        QG_TRY(make_map_i8(&tm.a[p], A + p * ps, kblocks, g.m_slot[0], BM));
        QG_TRY(make_map_i8(&tm.b[p], B + p * ps, kblocks, g.m_slot[b_slot], BN));
    }
    UnitsI8 u;
    u.ma = ma;
    u.nc = nc;
    u.ma_split = g.m_slot[0];
    u.mb_split = g.m_slot[b_slot];
    u.boff = b_off;
    u.tiles_m = (ma + BM - 1) / BM;
    u.tiles_n = (nc + BN - 1) / BN;
    u.lower = lower ? 1 : 0;
    u.ntiles = 0;
    for (int r = 0; r < u.tiles_m; ++r) u.ntiles += row_tiles(u, r);
    u.kblocks = (int)kblocks;
    const int G = sm_count_i8();
    u.nseg = std::max((u.kblocks + kSegMax - 1) / kSegMax, (4 * G + u.ntiles - 1) / u.ntiles);
    u.nseg = std::max(1, std::min(u.nseg, u.kblocks));
    u.kb_per_seg = (u.kblocks + u.nseg - 1) / u.nseg;
    u.nseg = (u.kblocks + u.kb_per_seg - 1) / u.kb_per_seg;
    u.units = u.ntiles * u.nseg;
    QG_TRY(g.part.reserve((size_t)u.units * BM * BN * sizeof(double)));
    const int grid = std::min(G, u.units);
    const size_t smem = 1024 + 1024 + (size_t)kStages * kStageBytes;
    QG_CUDA_TRY(allow_max_dynamic_smem(k_gram_i8));
    k_gram_i8<<<grid, kThreads, smem, st>>>(tm, u, g.part.as<double>(), err);
    QG_CUDA_TRY(cudaGetLastError());
    k_gram_i8_reduce<<<G * 4, 256, 0, st>>>(g.part.as<double>(), u, g.expo[0].as<int>(), g.expo[b_slot].as<int>(),
                                            alpha, C, ldc);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

}  // namespace

bool I8Gram::supported(long long N) { return N >= BK && encode_fn() != nullptr; }

long long I8Gram::kpad() const { return (N + BK - 1) / BK * BK; }

int I8Gram::setup(long long N_, int mmax_) {
    N = N_;
    mmax = mmax_;
    m_slot[0] = m_slot[1] = 0;
    return QG_OK;  // the slot buffers are allocated by the first split into them
}

int I8Gram::split(const double* A, int m, int which, cudaStream_t st) {
    if (m <= 0 || m > mmax || (which != 0 && which != 1)) return QG_ERR_INVALID;
    QG_TRY(slices[which].reserve((size_t)S * kpad() * mmax));
    QG_TRY(expo[which].reserve((size_t)mmax * sizeof(int)));
    k_col_expo<<<std::min(m, 148 * 4), 256, 0, st>>>(A, N, m, expo[which].as<int>());
    k_split_i8<<<148 * 8, 256, 0, st>>>(A, N, m, kpad(), expo[which].as<int>(), slices[which].as<int8_t>(),
                                        kpad() * mmax);
    QG_CUDA_TRY(cudaGetLastError());
    m_slot[which] = m;
    return QG_OK;
}

int I8Gram::gram(cudaStream_t st, int m, bool b_is_a, bool lower, double alpha, double* C, int ldc, int* err) {
    return run_i8(*this, st, m, m, b_is_a ? 0 : 1, 0, lower, alpha, C, ldc, err);
}

int I8Gram::gram_rect(cudaStream_t st, int ma, int nc, int b_slot, int b_off, double alpha, double* C, int ldc,
                      int* err) {
    return run_i8(*this, st, ma, nc, b_slot, b_off, false, alpha, C, ldc, err);
}

void I8Gram::release() {
    for (auto& b : slices) b.release();
    for (auto& b : expo) b.release();
    part.release();
}

}  // namespace qg
