// sfm_exec.cuh -- one cooperative launch for a whole ghost-fill-and-sweep
// sequence on the small fmg levels (blocks of 2^3 and 4^3 cells).
//
// On those levels a red-black colour of fmg_poisson_relax
// (fmg_poisson.F90:130-213) or vmg_poisson_relax (vmg_poisson.F90:114-141)
// is preceded by a converge_c2p of every AMR level, the ghost passes of
// fmg_ghostcell_fix (one per level and direction), the physical-boundary
// fill and the reflux -- some 25 short operations, each of which alone is a
// launch of a few microseconds over a few megabytes.  k_exec runs such a
// sequence (a "program" of phases built on the host) in one cooperative
// launch: every phase is the same per-element code as the separate kernels
// (the same functors and device functions), phases are separated by a grid
// barrier, so the results are bit-identical and the launch and ramp costs
// are paid once.
//
// The grid barrier spins a bounded number of times; a wait that gives up
// sets *err and the kernel returns (the host reports SFM_ETIMEOUT).  The
// launch is cooperative (all CTAs co-resident), so CTAs may wait on one
// another inside it.
#pragma once
#include "sfm_fast.cuh"

namespace sfm {

constexpr uint32_t kBarrierPolls = 1u << 22;
constexpr int kMaxPhases = 96;

struct GridBarrier {
    unsigned int count;
    unsigned int gen;
};

// all CTAs of the launch; false (and *err set) when the wait gave up
__device__ __forceinline__ bool grid_sync(GridBarrier *gb, int *err) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int *vgen = &gb->gen;
        const unsigned int g = *vgen;
        __threadfence();   // this CTA's writes (ordered by the barrier above) before the arrival
        int good = 1;
        if (atomicAdd(&gb->count, 1u) + 1u == gridDim.x) {
            atomicExch(&gb->count, 0u);
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else {
            for (uint32_t t = 0; *vgen == g; t++) {
                if (t >= kBarrierPolls) {
                    atomicExch(err, 1);
                    good = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();   // the other CTAs' writes before this CTA's next reads
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

enum : int8_t { PH_CONVERGE = 0, PH_GHOST = 1, PH_FILL0 = 2, PH_REFLUX = 3, PH_RELAX = 4 };

struct ExecPhase {
    int8_t kind, dir, sel, cubic;   // cubic: converge (cubic restriction) or ghost (bicubic)
    int32_t first, count;           // converge: first child block, children; ghost: face items;
                                    // fill0: boundary faces; reflux: reflux items
    int32_t ipass;                  // relax colour
    int32_t count0;                 // ghost: the first count0 items are same-level copies
};

template <class T>
struct ExecArgs {
    T *u;
    const T *rhs;
    const int32_t *parent;
    const int8_t *oct;
    const FaceItem *faces;
    const BFace *bfaces;
    const RefluxItem *reflux;
    double *rbuf;                    // reflux slots written by PH_REFLUX and read by PH_RELAX
    const double *h0;
    const int32_t *level;
    const int32_t *blocks;           // blocks swept by PH_RELAX
    int nblk;
    const int32_t *rslot;            // reflux slot per (block, face), or null (vmg)
    int f;
    unsigned long long *out;         // max |resh2| over the sweeps
    int *err;
    GridBarrier *gb;
    int nphase;
    ExecPhase ph[kMaxPhases];
};

template <class Op>
__device__ __forceinline__ void exec_elements(const Op &op, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) op(i);
}

template <class T, int N>
__global__ void __launch_bounds__(256) k_exec(const __grid_constant__ ExecArgs<T> a) {
    constexpr int G = N + 2, NB2 = N / 2, GT = N + 2;
    constexpr int64_t V = (int64_t)G * G * G;
    __shared__ GhostCubicTable<N> tab;
    __shared__ RelaxTileSmem<T, N> sm;
    constexpr bool kBicubicOk = NB2 + 2 >= 4;
    if (kBicubicOk && threadIdx.x < G)
        cubic_weights((int)threadIdx.x - 1, -1, NB2, tab.c[threadIdx.x], tab.w[threadIdx.x]);
    __syncthreads();
    constexpr int LN = ghost_lanes<N>();   // lanes per face item
    const int lane = threadIdx.x % LN;
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) / LN);
    const int nwarps = (int)((gridDim.x * blockDim.x) / LN);
    double m = 0.0;
    for (int p = 0; p < a.nphase; p++) {
        const ExecPhase ph = a.ph[p];
        switch (ph.kind) {
            case PH_CONVERGE:
                exec_elements(OpConverge<T>{a.u, a.parent, a.oct, ph.first, N, G, V, ph.cubic},
                              (int64_t)ph.count * NB2 * NB2 * NB2);
                break;
            case PH_GHOST: {
                // cells spread over the whole grid: a phase is small
                const int nc0 = ph.count0 * G * G, nthr = (int)(gridDim.x * blockDim.x);
                const int gt = (int)(blockIdx.x * blockDim.x + threadIdx.x);
                for (int b0 = 0; b0 < nc0; b0 += nthr * ghost_k<N>())
                    ghost_copy<T, N>(a.u, a.faces + ph.first, nc0, ph.dir, b0 + gt, nthr);
                const FaceItem *f1 = a.faces + ph.first + ph.count0;
                for (int it = warp; it < ph.count - ph.count0; it += nwarps)
                    ghost_face<T, N>(a.u, f1[it], ph.dir, ph.cubic && kBicubicOk, tab, lane);
                break;
            }
            case PH_FILL0:
                exec_elements(OpFill0Faces<T>{a.u, a.bfaces + ph.first, N, G, V}, (int64_t)ph.count * GT * GT);
                break;
            case PH_REFLUX:
                exec_elements(OpReflux<T>{a.u, a.reflux, a.rbuf, a.h0, a.level, a.f, N, G, V},
                              (int64_t)ph.count * NB2 * NB2);
                break;
            case PH_RELAX:
                relax_tiles<T, N>(sm, a.u, a.rhs, a.blocks, a.nblk, a.h0, a.level, a.rslot, a.rbuf, a.f, ph.ipass,
                                  blockIdx.x, gridDim.x, m);
                break;
        }
        if (p + 1 < a.nphase && !grid_sync(a.gb, a.err)) return;
    }
    cta_max_atomic(m, a.out);
}

}  // namespace sfm
