// Split-BF16 Gram products on the 5th-generation tensor cores (sm_100a):
//   C = alpha * A^T B,  A, B: N x m FP64 blocks (column-major, ld N)
// Each value is split into P bfloat16 pieces, a = a_0 + a_1 (+ a_2),
// a_0 = bf16(a), a_i = bf16(a - a_0 - ... - a_{i-1}), and the products a_i b_j
// with i + j < P are accumulated (P = 2: 3 products, ~2^-17 relative per
// product; P = 3: 6 products, ~2^-25).
//
// Persistent kernel, one CTA per SM, 10 warps:
//   warp 0      TMA producer: 128 x 64 bf16 tiles of every piece of A and B
//               (cp.async.bulk.tensor.2d, 128-byte swizzle) into a ring of S stages; the
//               pieces are stored K-block-major ([N / 64][m][64]), so each tile is one
//               contiguous 16 KB run (column-major pieces spread a tile over 128 columns
//               N * 2 bytes apart, which at N = 1.7 M halved the kernel's rate);
//   warp 1      owns 256 TMEM columns (two 128 x 128 FP32 accumulators); one lane
//               issues tcgen05.mma.cta_group::1.kind::f16 (M = N = 128, K = 16) for
//               every product and K step of a stage, then tcgen05.commit frees the
//               stage and hands the accumulator to the epilogue;
//   warps 2-9   epilogue: tcgen05.ld of the accumulator after every 64-row K block
//               (3 pieces; every second block for 2 pieces), added into FP64 registers
//               (each thread: one tile row, 64 columns), so the FP32 accumulation spans
//               64 (128) rows only (the tensor cores' FP32 sums drift on long same-sign
//               runs); the accumulator buffers alternate so the MMAs of the next block
//               overlap the read-out of the last.
// Work units are (tile, K segment), K-segment-major so that concurrent CTAs stream
// the same rows of A and B (L2 reuse); every unit writes its FP64 partial tile once,
// and k_gram_reduce sums the segments in a fixed order (deterministic).
// Every mbarrier wait is bounded; on timeout the kernel records QG_ERR_TIMEOUT,
// all roles stop, the MMAs already issued are waited for, and TMEM is released.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "gram_tc.h"
#include "tc_common.cuh"

namespace qg {
namespace {

using namespace tc;
using tchost::EncodeTiledFn;
using tchost::encode_fn;

constexpr int BM = 128, BK = 64;
constexpr int kThreads = 320;
constexpr int kTileBytes = BM * BK * 2;  // 16 KB per piece tile
constexpr int kEpiWarps = 8;
constexpr int kAccCols = 128;
// 64-row K blocks summed in FP32 (TMEM) between read-outs: 2 for the 2-piece split
// (47.6 against 56.4 ms at N = 1.728 M x 1584, error unchanged at its 2^-18 level), 1 for
// the 3-piece split (the same 79 ms either way, while 2 doubles its FP32 drift on
// norm-like entries to 1.4e-6)
template <int P>
constexpr int readout_blocks() { return P == 2 ? 2 : 1; }

struct TMaps {
    CUtensorMap a[3];
    CUtensorMap b[3];
};

struct Units {
    int tiles_m;     // 128-row tiles along m
    int ntiles;      // tiles computed (lower triangle or all)
    int lower;
    int nseg;        // K segments
    int kblocks;     // ceil(N / 64)
    int kb_per_seg;
    int units;       // ntiles * nseg
    int m;
};

// Shared-memory matrix descriptor of a K-major 128 x 64 bf16 tile written by TMA
// with the 128-byte swizzle: 8-row core groups 1024 bytes apart (SBO), descriptor
// version 1, layout type 2 (SWIZZLE_128B); the K step of 16 elements advances the
// start address by 32 bytes.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFF) >> 4) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both K-major,
// N = 128 (n_dim = N >> 3 at bit 17), M = 128 (m_dim = M >> 4 at bit 24).
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void unit_coords(int unit, const Units& u, int& seg, int& ti, int& tj) {
    seg = unit / u.ntiles;
    const int t = unit - seg * u.ntiles;
    if (u.lower) {
        int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
        while ((i + 1) * (i + 2) / 2 <= t) ++i;
        while (i * (i + 1) / 2 > t) --i;
        ti = i;
        tj = t - i * (i + 1) / 2;
    } else {
        ti = t / u.tiles_m;
        tj = t - ti * u.tiles_m;
    }
}

template <int P>
struct Products;
template <>
struct Products<2> {
    static constexpr int n = 3;
    __device__ static constexpr int a(int k) { return k == 2 ? 1 : 0; }
    __device__ static constexpr int b(int k) { return k == 1 ? 1 : 0; }
};
template <>
struct Products<3> {
    static constexpr int n = 6;  // (0,0) (0,1) (1,0) (0,2) (1,1) (2,0)
    __device__ static constexpr int a(int k) { return k == 2 ? 1 : (k == 4 ? 1 : (k == 5 ? 2 : 0)); }
    __device__ static constexpr int b(int k) { return k == 1 ? 1 : (k == 3 ? 2 : (k == 4 ? 1 : 0)); }
};

template <int P, int S>
__global__ void __launch_bounds__(kThreads, 1)
    k_gram_tc(const __grid_constant__ TMaps tm, const Units u, double* __restrict__ part, int* err) {
    extern __shared__ unsigned char smem_raw[];
    // 1024-byte aligned base for the swizzled tiles
    unsigned char* base = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = reinterpret_cast<uint64_t*>(base);
    uint64_t* empty = full + S;
    uint64_t* accfull = empty + S;
    uint64_t* accempty = accfull + 2;
    uint64_t* done = accempty + 2;
    volatile uint32_t* tmem_slot = reinterpret_cast<volatile uint32_t*>(done + 1);
    volatile int* ctl = reinterpret_cast<volatile int*>(tmem_slot + 1);
    unsigned char* tiles = base + 1024;
    constexpr int kStageBytes = 2 * P * kTileBytes;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < S; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&accfull[i], 1);
            mbar_init(&accempty[i], kEpiWarps);
        }
        mbar_init(done, 1);
        ctl[0] = 0;
        ctl[1] = -1;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32((const void*)tmem_slot)),
                     "r"(2 * kAccCols)
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
                int seg, ti, tj;
                unit_coords(unit, u, seg, ti, tj);
                const int kb0 = seg * u.kb_per_seg, kb1 = min(u.kblocks, kb0 + u.kb_per_seg);
                for (int kb = kb0; kb < kb1; ++kb, ++pos) {
                    const int j = pos % S, k = pos / S;
                    if (k > 0 && !mbar_wait(&empty[j], (uint32_t)(k - 1) & 1u)) {
                        ctl[0] = 1;
                        atomicExch(err, (int)QG_ERR_TIMEOUT);
                        break;
                    }
                    if (ctl[0]) break;
                    unsigned char* st = tiles + (size_t)j * kStageBytes;
                    mbar_expect_tx(&full[j], kStageBytes);
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                        // pieces are K-block-major: block kb holds the 64-row segments of all
                        // m columns, so a 128-column tile is one contiguous 16 KB run
                        tma_load_2d(st + p * kTileBytes, &tm.a[p], 0, kb * u.m + ti * BM, &full[j]);
                        tma_load_2d(st + (P + p) * kTileBytes, &tm.b[p], 0, kb * u.m + tj * BM, &full[j]);
                    }
                    ctl[1] = pos;
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int pos = 0, accpos = 0;
            for (int unit = blockIdx.x; unit < u.units && !ctl[0]; unit += gridDim.x) {
                int seg, ti, tj;
                unit_coords(unit, u, seg, ti, tj);
                const int kb0 = seg * u.kb_per_seg, kb1 = min(u.kblocks, kb0 + u.kb_per_seg);
                for (int kb = kb0; kb < kb1; ++kb, ++pos) {
                    const int j = pos % S, k = pos / S;
                    const int buf = accpos & 1, n = accpos >> 1;
                    constexpr int RO = readout_blocks<P>();
                    const bool first = (kb - kb0) % RO == 0;
                    const bool last = (kb - kb0) % RO == RO - 1 || kb == kb1 - 1;
                    bool ok = mbar_wait(&full[j], (uint32_t)k & 1u);
                    if (ok && first && n > 0) ok = mbar_wait(&accempty[buf], (uint32_t)(n - 1) & 1u);
                    if (!ok || ctl[0]) {
                        ctl[0] = 1;
                        if (!ok) atomicExch(err, (int)QG_ERR_TIMEOUT);
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = smem_u32(tiles + (size_t)j * kStageBytes);
                    const uint32_t d = tmem + (uint32_t)(buf * kAccCols);
#pragma unroll
                    for (int kk = 0; kk < BK / 16; ++kk) {
#pragma unroll
                        for (int q = 0; q < Products<P>::n; ++q) {
                            const uint64_t ad = sw128_desc(st + Products<P>::a(q) * kTileBytes) + 2 * kk;
                            const uint64_t bd = sw128_desc(st + (P + Products<P>::b(q)) * kTileBytes) + 2 * kk;
                            umma_f16(d, ad, bd, (!first || kk || q) ? 1u : 0u);
                        }
                    }
                    umma_commit(&empty[j]);  // the stage is free once these MMAs have read it
                    if (last) {
                        umma_commit(&accfull[buf]);  // the accumulator holds this group of K blocks
                        ++accpos;
                    }
                }
            }
            umma_commit(done);  // completes once every MMA issued above has finished
            mbar_wait(done, 0);
        }
    } else {
        // ---------------- epilogue: TMEM -> FP64 registers ----------------
        const int lg = warp & 3;                  // TMEM lane group this warp may read
        const int half = (warp - 2) >> 2;         // column half of the tile
        const int row = lg * 32 + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(lg * 32) << 16) + (uint32_t)(half * 64);
        double acc[64];
#pragma unroll
        for (int i = 0; i < 64; ++i) acc[i] = 0.0;
        int accpos = 0;
        bool bad = false;
        for (int unit = blockIdx.x; unit < u.units && !bad; unit += gridDim.x) {
            int seg, ti, tj;
            unit_coords(unit, u, seg, ti, tj);
            const int kb0 = seg * u.kb_per_seg, kb1 = min(u.kblocks, kb0 + u.kb_per_seg);
            for (int kb = kb0; kb < kb1; kb += readout_blocks<P>(), ++accpos) {
                const int buf = accpos & 1, n = accpos >> 1;
                const bool ok = mbar_wait(&accfull[buf], (uint32_t)n & 1u);
                if (__any_sync(0xffffffffu, !ok || ctl[0] != 0)) {
                    bad = true;
                    break;
                }
                tc_fence_after();
                uint32_t r[32];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    tmem_ld32(lane_addr + (uint32_t)(buf * kAccCols + h * 32), r);
                    tmem_wait_ld();
#pragma unroll
                    for (int i = 0; i < 32; ++i) acc[h * 32 + i] += (double)__uint_as_float(r[i]);
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&accempty[buf]);
            }
            if (bad) break;
            // this unit's FP64 partial tile: part[(seg * ntiles + t)][row][col], 128 x 128
            double* dst = part + (size_t)unit * (BM * BM) + (size_t)row * BM + half * 64;
#pragma unroll
            for (int i = 0; i < 64; i += 2) {
                *reinterpret_cast<double2*>(dst + i) = make_double2(acc[i], acc[i + 1]);
                acc[i] = 0.0;
                acc[i + 1] = 0.0;
            }
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
        for (int ps = max(0, last - S + 1); ps <= last; ++ps) mbar_wait(&full[ps % S], (uint32_t)(ps / S) & 1u);
    }
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kAccCols)
                     : "memory");
    }
}

// C(i, j) = alpha * sum_seg part[seg][tile(i, j)][i % 128][j % 128], C column-major (ld ldc);
// lower: only the tiles of the lower triangle (ti >= tj). Threads walk the partial tiles
// contiguously (the segments' reads are coalesced); the segments add in order.
__global__ void k_gram_reduce(const double* __restrict__ part, Units u, double alpha, double* __restrict__ C,
                              int ldc) {
    const long long total = (long long)u.ntiles * (BM * BM);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
        const int t = (int)(e / (BM * BM));
        const int off = (int)(e - (long long)t * (BM * BM));
        int seg, ti, tj;
        unit_coords(t, u, seg, ti, tj);
        const int i = ti * BM + off / BM, j = tj * BM + off % BM;
        if (i >= u.m || j >= u.m) continue;
        double s = 0.0;
        for (int sg = 0; sg < u.nseg; ++sg) s += part[((size_t)sg * u.ntiles + t) * (BM * BM) + off];
        C[i + (long long)j * ldc] = alpha * s;
    }
}

// The P bf16 pieces of the N x m block src (column-major, ld N), K-block-major:
// dst[p][((k / 64) * m + j) * 64 + k % 64] for row k and column j, rows N .. kpad-1 of the
// last block zero (kpad = N rounded up to 64).
template <int P>
__global__ void k_split_pieces(const double* __restrict__ src, long long N, int m, long long kpad,
                               __nv_bfloat16* __restrict__ dst, long long piece_stride) {
    const long long n = kpad * m;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const long long blk = i >> 6;  // (k / 64) * m + j
        const int r = (int)(i & 63);
        const long long kb = blk / m;
        const int j = (int)(blk - kb * m);
        const long long k = kb * BK + r;
        double v = k < N ? src[(long long)j * N + k] : 0.0;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const __nv_bfloat16 h = __double2bfloat16(v);
            dst[p * piece_stride + i] = h;
            v -= (double)__bfloat162float(h);
        }
    }
}

int make_map(CUtensorMap* map, const __nv_bfloat16* ptr, long long kblocks, int m) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return QG_ERR_UNSUPPORTED;
    const cuuint64_t dims[2] = {(cuuint64_t)BK, (cuuint64_t)(kblocks * m)};
    const cuuint64_t strides[1] = {(cuuint64_t)BK * 2};
    const cuuint32_t box[2] = {BK, BM};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult rc = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(ptr), dims, strides,
                            box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return rc == CUDA_SUCCESS ? QG_OK : QG_ERR_UNSUPPORTED;
}

template <int P>
constexpr int stages() { return P == 2 ? 3 : 2; }

template <int P>
size_t smem_bytes() { return 1024 + 1024 + (size_t)stages<P>() * 2 * P * kTileBytes; }

int sm_count_dev() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

}  // namespace

bool TcGram::supported(long long N) { return N >= BK && encode_fn() != nullptr; }

long long TcGram::kpad() const { return (N + BK - 1) / BK * BK; }

int TcGram::setup(long long N_, int mmax_, int pieces_) {
    if (pieces_ != 2 && pieces_ != 3) return QG_ERR_INVALID;
    N = N_;
    mmax = mmax_;
    pieces = pieces_;
    QG_TRY(split_a.reserve((size_t)pieces * kpad() * mmax * sizeof(__nv_bfloat16)));
    return QG_OK;  // the B-side slot is allocated by the first split into it
}

int TcGram::split(const double* A, int m, int which, cudaStream_t st) {
    DevBuf& b = which == 0 ? split_a : split_b;
    if (m <= 0 || m > mmax) return QG_ERR_INVALID;
    QG_TRY(b.reserve((size_t)pieces * kpad() * mmax * sizeof(__nv_bfloat16)));
    const long long ps = kpad() * mmax;
    if (pieces == 2)
        k_split_pieces<2><<<148 * 8, 256, 0, st>>>(A, N, m, kpad(), b.as<__nv_bfloat16>(), ps);
    else
        k_split_pieces<3><<<148 * 8, 256, 0, st>>>(A, N, m, kpad(), b.as<__nv_bfloat16>(), ps);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

int TcGram::gram(cudaStream_t st, int m, bool b_is_a, bool lower, double alpha, double* C, int ldc, int* err) {
    TMaps tm;
    std::memset(&tm, 0, sizeof(tm));
    const __nv_bfloat16* A = split_a.as<__nv_bfloat16>();
    const __nv_bfloat16* B = b_is_a ? A : split_b.as<__nv_bfloat16>();
    if (m <= 0 || m > mmax) return QG_ERR_INVALID;
    const long long ps = kpad() * mmax;
    for (int p = 0; p < pieces; ++p) {
        QG_TRY(make_map(&tm.a[p], A + p * ps, kpad() / BK, m));
        QG_TRY(make_map(&tm.b[p], B + p * ps, kpad() / BK, m));
    }
    Units u;
    u.m = m;
    u.tiles_m = (m + BM - 1) / BM;
    u.lower = lower ? 1 : 0;
    u.ntiles = lower ? u.tiles_m * (u.tiles_m + 1) / 2 : u.tiles_m * u.tiles_m;
    u.kblocks = (int)((N + BK - 1) / BK);
    const int G = sm_count_dev();
    u.nseg = std::max(1, std::min(u.kblocks, (4 * G + u.ntiles - 1) / u.ntiles));
    u.kb_per_seg = (u.kblocks + u.nseg - 1) / u.nseg;
    u.nseg = (u.kblocks + u.kb_per_seg - 1) / u.kb_per_seg;
    u.units = u.ntiles * u.nseg;
    QG_TRY(part.reserve((size_t)u.units * BM * BM * sizeof(double)));
    const int grid = std::min(G, u.units);
    if (pieces == 2) {
        auto kern = k_gram_tc<2, stages<2>()>;
        const size_t sm = smem_bytes<2>();
        QG_CUDA_TRY(allow_max_dynamic_smem(kern));
        kern<<<grid, kThreads, sm, st>>>(tm, u, part.as<double>(), err);
    } else {
        auto kern = k_gram_tc<3, stages<3>()>;
        const size_t sm = smem_bytes<3>();
        QG_CUDA_TRY(allow_max_dynamic_smem(kern));
        kern<<<grid, kThreads, sm, st>>>(tm, u, part.as<double>(), err);
    }
    QG_CUDA_TRY(cudaGetLastError());
    k_gram_reduce<<<G * 4, 256, 0, st>>>(part.as<double>(), u, alpha, C, ldc);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

void TcGram::release() {
    split_a.release();
    split_b.release();
    part.release();
}

}  // namespace qg
