// FD stencil + local potential, H psi = V psi - 1/2 Lap psi, two output planes per
// consumer step (real states, sm_100a).
//
// Same plane ring as k_stencil_tma (a producer lane streams each work item's planes
// with bulk async copies into shared-memory stages counted on mbarriers; consumer
// warps release stages through "empty" mbarriers; work item = (state, y tile of ty
// full x-rows, z slab), one persistent block per SM), but each consumer step
// produces two consecutive z-planes:
//  * one pair of ring waits, one warp vote and one index update per two planes, and
//    two planes' shared-memory loads and FP64 sums in flight between them (twice
//    the independent work per synchronisation point of the one-plane kernel, whose
//    consumers stall on shared-memory and barrier latency at 14 warps per SM);
//  * the thread's z-window holds planes z-R .. z+1+R (2R+2 values per x-point) in
//    registers; the step loop is unrolled over the window's renaming period, so the
//    window rotates by renaming, not by register moves;
//  * V of the two output planes is prefetched two steps ahead from global memory.
// Each point's sum is the Laplacian grouping of Laplasian{2nd,4th,6th,8th}_halo_f
// (GridDifference2nd.h:1027-1031, 4th.h:528-530, 6th.h:425-429, 8th.h:141-145),
// with each axis' sum formed independently and then added in x, y, z order.
// Every mbarrier wait is bounded; on timeout the thread records QG_ERR_TIMEOUT in the
// device status word, the block winds down and the producer waits (bounded) for its
// copies in flight.
#include <cstdint>

#include "qg_internal.h"
#include "stencil_common.cuh"
#include "tma_ring.cuh"

namespace qg {
namespace {

using namespace ring;

constexpr int kPairThreads = 352;    // one producer warp + up to 320 consumer threads
constexpr int kPairConsumers = 320;  // (184 registers per thread at one block per SM)

template <int ORDER>
constexpr int pair_radius() { return ORDER == 2 ? 1 : (ORDER == 8 ? 4 : 3); }

// 16-byte vector <-> PX scalars
template <typename T>
struct V16;
template <>
struct V16<double> {
    static constexpr int n = 2;
    static __device__ __forceinline__ void ld(double (&v)[2], const double* p) {
        const double2 w = *reinterpret_cast<const double2*>(p);
        v[0] = w.x; v[1] = w.y;
    }
    static __device__ __forceinline__ void ldg(double (&v)[2], const double* p) {
        const double2 w = __ldg(reinterpret_cast<const double2*>(p));
        v[0] = w.x; v[1] = w.y;
    }
    static __device__ __forceinline__ void st(double* p, const double (&v)[2]) {
        *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
    }
};
template <>
struct V16<float> {
    static constexpr int n = 4;
    static __device__ __forceinline__ void ld(float (&v)[4], const float* p) {
        const float4 w = *reinterpret_cast<const float4*>(p);
        v[0] = w.x; v[1] = w.y; v[2] = w.z; v[3] = w.w;
    }
    static __device__ __forceinline__ void ldg(float (&v)[4], const float* p) {
        const float4 w = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = w.x; v[1] = w.y; v[2] = w.z; v[3] = w.w;
    }
    static __device__ __forceinline__ void st(float* p, const float (&v)[4]) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
};

// -1/2 Lap at one point: xm[d]/xp[d] = psi at x -/+ (d+1), same for y and z; each
// axis sum is independent, then c0*c + Sx + Sy + Sz (orders 6, 8) or Sx + Sy + Sz.
template <typename T, int ORDER>
__device__ __forceinline__ T lap_axes(T c, const T* xm, const T* xp, const T* ym, const T* yp, const T* zm,
                                      const T* zp, const HamArgs<T>& a) {
    if constexpr (ORDER == 2) {
        return a.cx[0] * (xp[0] + xm[0] - T(2) * c) + a.cy[0] * (yp[0] + ym[0] - T(2) * c) +
               a.cz[0] * (zp[0] + zm[0] - T(2) * c);
    } else if constexpr (ORDER == 4) {
        return a.cx[2] * ((xp[2] + xm[2]) - T(54) * (xp[1] + xm[1]) + T(783) * (xp[0] + xm[0]) - T(1460) * c) +
               a.cy[2] * ((yp[2] + ym[2]) - T(54) * (yp[1] + ym[1]) + T(783) * (yp[0] + ym[0]) - T(1460) * c) +
               a.cz[2] * ((zp[2] + zm[2]) - T(54) * (zp[1] + zm[1]) + T(783) * (zp[0] + zm[0]) - T(1460) * c);
    } else if constexpr (ORDER == 6) {
        const T sx = a.cx[2] * (xp[2] + xm[2]) + a.cx[1] * (xp[1] + xm[1]) + a.cx[0] * (xp[0] + xm[0]);
        const T sy = a.cy[2] * (yp[2] + ym[2]) + a.cy[1] * (yp[1] + ym[1]) + a.cy[0] * (yp[0] + ym[0]);
        const T sz = a.cz[2] * (zp[2] + zm[2]) + a.cz[1] * (zp[1] + zm[1]) + a.cz[0] * (zp[0] + zm[0]);
        return ((a.c0 * c + sx) + sy) + sz;
    } else {
        const T sx = a.cx[3] * (xp[3] + xm[3]) + a.cx[2] * (xp[2] + xm[2]) + a.cx[1] * (xp[1] + xm[1]) +
                     a.cx[0] * (xp[0] + xm[0]);
        const T sy = a.cy[3] * (yp[3] + ym[3]) + a.cy[2] * (yp[2] + ym[2]) + a.cy[1] * (yp[1] + ym[1]) +
                     a.cy[0] * (yp[0] + ym[0]);
        const T sz = a.cz[3] * (zp[3] + zm[3]) + a.cz[2] * (zp[2] + zm[2]) + a.cz[1] * (zp[1] + zm[1]) +
                     a.cz[0] * (zp[0] + zm[0]);
        return ((a.c0 * c + sx) + sy) + sz;
    }
}

template <typename T, int ORDER, int NXC>
__global__ void __launch_bounds__(kPairThreads, 1) k_stencil_pair(const HamArgs<T> a, const WorkGrid wg, int nst) {
    constexpr int PX = 16 / sizeof(T);
    constexpr int R = pair_radius<ORDER>();
    constexpr int ZB = 2;            // output planes per step
    constexpr int W = 2 * R + ZB;    // z-window length (planes z-R .. z+1+R)
    constexpr int P = W / ZB;        // renaming period in steps (W is even)
    constexpr int NV = (R + PX - 1) / PX;
    using VV = V16<T>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + nst;
    volatile int* ctl = reinterpret_cast<volatile int*>(empty + nst);  // [0] abort, [1] last position issued
    T* ringp = reinterpret_cast<T*>(smem + kBarBytes);

    const int nx = NXC > 0 ? NXC : a.nx, ny = a.ny, nz = a.nz, ty = a.ty;
    const int rows = ty + 2 * R;
    const int stage_elems = rows * nx;
    const int tpr = nx / PX;
    const int ncons = tpr * ty;
    const int ncons_warps = (ncons + 31) / 32;
    const int t = threadIdx.x;
    const long long plane = (long long)nx * ny;

    if (t == 0) {
        for (int i = 0; i < nst; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], (uint32_t)ncons_warps);
        }
        ctl[0] = 0;
        ctl[1] = -1;
        fence_mbar_init();
    }
    __syncthreads();

    if (t < 32) {
        if (t == 0) produce_planes<T, R, 1>(a, wg, nst, nx, ringp, full, empty, ctl);
    } else if (t < 32 + ncons) {
        const unsigned wmask = __activemask();
        const int lane = t & 31;
        const int c = t - 32;
        const int ix0 = (c % tpr) * PX;
        const int ly = c / tpr;
        const int cb = (R + ly) * nx + ix0;  // the thread's first point inside a stage
        int xo[2 * NV];                      // x-neighbour vectors (wrapped in x) inside a stage
#pragma unroll
        for (int v = 0; v < 2 * NV; ++v) {
            const int dv = (v < NV) ? (v - NV) : (v - NV + 1);
            int xx = ix0 + dv * PX;
            xx += (xx < 0) ? nx : 0;
            xx -= (xx >= nx) ? nx : 0;
            xo[v] = (R + ly) * nx + xx;
        }
        int pos = 0;
        bool bad = false;
        for (int item = blockIdx.x; item < wg.items && !bad; item += gridDim.x) {
            const int slab = item % wg.nslab;
            const int tile = (item / wg.nslab) % wg.tiles;
            const int s = item / (wg.nslab * wg.tiles);
            const int iy = tile * ty + ly;
            const int zs = slab * wg.zslab;
            const int ze = min(nz, zs + wg.zslab);
            const long long col = (long long)iy * nx + ix0;

            // z-window: plane z - R + d in slot (ZB*k + d) % W at unrolled step k
            T q[W][PX];
            int j = pos % nst;
            uint32_t ph = (uint32_t)(pos / nst) & 1u;
            bool w = true;
#pragma unroll
            for (int d = 0; d < 2 * R; ++d) {  // planes zs-R .. zs+R-1
                if (w && !mbar_wait(&full[j], ph)) w = false;
                VV::ld(q[d], ringp + j * stage_elems + cb);
                if (++j == nst) { j = 0; ph ^= 1u; }
            }
            const T* vcol = a.V + col;
            T vc[ZB][PX], vn[ZB][PX];
#pragma unroll
            for (int p = 0; p < ZB; ++p) {
#pragma unroll
                for (int e = 0; e < PX; ++e) vc[p][e] = vn[p][e] = T(0);
                if (zs + p < ze) VV::ldg(vc[p], vcol + (long long)(zs + p) * plane);
                if (zs + ZB + p < ze) VV::ldg(vn[p], vcol + (long long)(zs + ZB + p) * plane);
            }
            if (__any_sync(wmask, !w)) {
                bad = true;
                break;
            }
            __syncwarp(wmask);
            int jz = pos % nst;
            if (lane == 0)
                for (int d = 0; d < R; ++d) {  // planes zs-R .. zs-1 live on in registers only
                    mbar_arrive(&empty[jz]);
                    if (++jz == nst) jz = 0;
                }
            jz = (pos + R) % nst;  // stage of plane z
            int jp = j;            // stage of plane z + R
            uint32_t php = ph;
            T* hcol = a.HX + state_offset(a, s, true) + col;
            for (int z = zs; z < ze && !bad;) {
#pragma unroll
                for (int k = 0; k < P; ++k) {
                    if (z >= ze) break;
                    const bool two = z + 1 < ze;
                    int jp1 = jp + 1;
                    uint32_t php1 = php;
                    if (jp1 == nst) { jp1 = 0; php1 ^= 1u; }
                    bool ok = mbar_wait(&full[jp], php);
                    if (two && ok) ok = mbar_wait(&full[jp1], php1);
                    if (__any_sync(wmask, !ok)) {
                        bad = true;
                        break;
                    }
                    VV::ld(q[(ZB * k + 2 * R) % W], ringp + jp * stage_elems + cb);
                    if (two) VV::ld(q[(ZB * k + 2 * R + 1) % W], ringp + jp1 * stage_elems + cb);
                    int jz1 = jz + 1;
                    if (jz1 == nst) jz1 = 0;
                    T out[ZB][PX];
#pragma unroll
                    for (int p = 0; p < ZB; ++p) {
                        if (p > 0 && !two) break;
                        const T* st = ringp + (p ? jz1 : jz) * stage_elems;
                        const int cs = (ZB * k + p + R) % W;  // centre slot
                        T xv[(2 * NV + 1) * PX];
#pragma unroll
                        for (int v = 0; v < 2 * NV; ++v) {
                            T tv[PX];
                            VV::ld(tv, st + xo[v]);
                            const int slot = (v < NV) ? v : v + 1;
#pragma unroll
                            for (int e = 0; e < PX; ++e) xv[slot * PX + e] = tv[e];
                        }
#pragma unroll
                        for (int e = 0; e < PX; ++e) xv[NV * PX + e] = q[cs][e];
                        T ypv[R][PX], ymv[R][PX];
#pragma unroll
                        for (int d = 1; d <= R; ++d) {
                            VV::ld(ypv[d - 1], st + cb + d * nx);
                            VV::ld(ymv[d - 1], st + cb - d * nx);
                        }
#pragma unroll
                        for (int e = 0; e < PX; ++e) {
                            T xm[R], xp[R], ym[R], yp[R], zm[R], zp[R];
#pragma unroll
                            for (int d = 1; d <= R; ++d) {
                                xm[d - 1] = xv[NV * PX + e - d];
                                xp[d - 1] = xv[NV * PX + e + d];
                                ym[d - 1] = ymv[d - 1][e];
                                yp[d - 1] = ypv[d - 1][e];
                                zm[d - 1] = q[(ZB * k + p + R - d) % W][e];
                                zp[d - 1] = q[(ZB * k + p + R + d) % W][e];
                            }
                            const T lap = lap_axes<T, ORDER>(q[cs][e], xm, xp, ym, yp, zm, zp, a);
                            out[p][e] = vc[p][e] * q[cs][e] + lap;
                        }
                    }
                    VV::st(hcol + (long long)z * plane, out[0]);
                    if (two) VV::st(hcol + (long long)(z + 1) * plane, out[1]);
                    __syncwarp(wmask);
                    if (lane == 0) {  // planes z (and z+1) are no longer read
                        mbar_arrive(&empty[jz]);
                        if (two) mbar_arrive(&empty[jz1]);
                    }
                    const int adv = two ? 2 : 1;
                    z += adv;
                    jz += adv;
                    if (jz >= nst) jz -= nst;
                    jp += adv;
                    if (jp >= nst) { jp -= nst; php ^= 1u; }
                    // V: the next step's planes move in, the one after is prefetched
#pragma unroll
                    for (int p = 0; p < ZB; ++p) {
#pragma unroll
                        for (int e = 0; e < PX; ++e) vc[p][e] = vn[p][e];
                        if (z + ZB + p < ze) VV::ldg(vn[p], vcol + (long long)(z + ZB + p) * plane);
                    }
                }
            }
            if (bad) break;
            __syncwarp(wmask);
            if (lane == 0)
                for (int d = 0; d < R; ++d) {  // planes ze .. ze+R-1
                    mbar_arrive(&empty[jz]);
                    if (++jz == nst) jz = 0;
                }
            pos += ze - zs + 2 * R;
        }
        if (bad) {
            ctl[0] = 1;
            if (lane == 0) atomicExch(a.err, (int)QG_ERR_TIMEOUT);
        }
    }
    __syncthreads();
    if (t == 0 && ctl[0]) {
        // wind down: wait (bounded) for the fills still in flight
        const int last = ctl[1];
        for (int ps = max(0, last - nst + 1); ps <= last; ++ps) mbar_wait(&full[ps % nst], (uint32_t)(ps / nst) & 1u);
    }
}

// Rows per tile: the largest divisor of ny (<= 16) keeping the consumers within the limit.
int pair_tile_rows(int nx, int ny, int px) {
    int ty = 0;
    for (int t = 1; t <= 16; ++t)
        if (ny % t == 0 && (nx / px) * t <= kPairConsumers) ty = t;
    return ty;
}

template <typename T, int ORDER, int NXC = 0>
int launch_pair_order(const HamArgs<T>& a, cudaStream_t st) {
    constexpr int PX = 16 / sizeof(T);
    constexpr int R = pair_radius<ORDER>();
    if constexpr (NXC == 0) {
        switch (a.nx) {
            case 40: return launch_pair_order<T, ORDER, 40>(a, st);
            case 80: return launch_pair_order<T, ORDER, 80>(a, st);
            case 120: return launch_pair_order<T, ORDER, 120>(a, st);
            default: break;
        }
    }
    const size_t stage = (size_t)(a.ty + 2 * R) * a.nx * sizeof(T);
    const int nst = ring_stages(R, stage, 3);
    if (nst < 0) return QG_ERR_UNSUPPORTED;
    const size_t smem = kBarBytes + (size_t)nst * stage;
    auto kern = k_stencil_pair<T, ORDER, NXC>;
    if (allow_max_dynamic_smem(kern) != cudaSuccess)
        return QG_ERR_UNSUPPORTED;
    const int ncons = (a.nx / PX) * a.ty;
    const int threads = 32 + ncons;
    if (threads > kPairThreads) return QG_ERR_UNSUPPORTED;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
        return QG_ERR_UNSUPPORTED;
    const int G0 = sm_count() * per_sm;
    WorkGrid wg;
    wg.tiles = a.ny / a.ty;
    const long long base = (long long)a.ns * wg.tiles;
    wg.nslab = 1;
    while (base * wg.nslab < 4LL * G0 && a.nz / (wg.nslab * 2) >= 2 * R) wg.nslab *= 2;
    wg.zslab = (a.nz + wg.nslab - 1) / wg.nslab;
    wg.nslab = (a.nz + wg.zslab - 1) / wg.zslab;
    wg.items = (int)(base * wg.nslab);
    const int G = std::min(G0, wg.items);
    kern<<<G, threads, smem, st>>>(a, wg, nst);
    return QG_OK;
}

}  // namespace

template <typename T>
bool stencil_pair_ok(const HamArgs<T>& a, int order) {
    constexpr int PX = 16 / sizeof(T);
    const int R = order == 2 ? 1 : (order == 8 ? 4 : 3);
    if (order != 2 && order != 4 && order != 6 && order != 8) return false;
    if (a.row) return false;
    if (a.nsk > 0) return false;
    if (a.nx % PX != 0 || ((uintptr_t)a.X % 16) || ((uintptr_t)a.HX % 16) || ((uintptr_t)a.V % 16) ||
        (a.ldx % PX) || (a.ldhx % PX) || !a.err || a.ny < 2 * R || a.nx < 2 * R || a.nz < 2 * R)
        return false;
    const int ty = pair_tile_rows(a.nx, a.ny, PX);
    if (ty == 0) return false;
    return ring_stages(R, (size_t)(ty + 2 * R) * a.nx * sizeof(T), 3) > 0;
}

template <typename T>
int launch_stencil_pair(const HamArgs<T>& a, int order, cudaStream_t st) {
    if (!stencil_pair_ok<T>(a, order)) return QG_ERR_UNSUPPORTED;
    HamArgs<T> b = a;
    b.ty = pair_tile_rows(a.nx, a.ny, 16 / sizeof(T));
    switch (order) {
        case 2: return launch_pair_order<T, 2>(b, st);
        case 4: return launch_pair_order<T, 4>(b, st);
        case 6: return launch_pair_order<T, 6>(b, st);
        case 8: return launch_pair_order<T, 8>(b, st);
        default: return QG_ERR_INVALID;
    }
}

template bool stencil_pair_ok<double>(const HamArgs<double>&, int);
template bool stencil_pair_ok<float>(const HamArgs<float>&, int);
template int launch_stencil_pair<double>(const HamArgs<double>&, int, cudaStream_t);
template int launch_stencil_pair<float>(const HamArgs<float>&, int, cudaStream_t);

}  // namespace qg
