// sfm_fast.cuh -- block-tiled kernels for the hot operations.
//
// These replace the per-element functors for the operations that dominate a
// solve (ghost passes, red-black colour sweeps, residuals, restriction and
// prolongation).  Each evaluates exactly the same expressions in the same
// order as the functors of sfm_device.cuh (and as the reference), so FP64
// results stay bit-identical; what changes is the work decomposition:
//   - ghost passes: one warp per block face, compile-time index math;
//   - smoother / residual: one CTA per block (or several small blocks), the
//     block with its ghost shell staged in shared memory by coalesced loads,
//     updated values written back as whole interior rows;
//   - prolongation: the separable tricubic of interp_tricubic staged in
//     shared memory per block, as the reference stages bufx/bufxy.
#pragma once
#include "sfm_device.cuh"

namespace sfm {

// ---------------------------------------------------------------------------
// ghost pass: one warp per face item
// ---------------------------------------------------------------------------
// transverse Lagrange nodes and weights of the bicubic coarse-fine ghost for
// p in [-1, N] (entry p + 1), built once per CTA by its first G threads
template <int N>
struct GhostCubicTable {
    int c[N + 2][4];
    double w[N + 2][4];
};

// lanes serving one face: a 2^3 block's face has 16 ghost cells, so a warp
// serves two of them
template <int N>
__host__ __device__ constexpr int ghost_lanes() { return (N + 2) * (N + 2) <= 16 ? 16 : 32; }

// one face item, by ghost_lanes<N>() lanes (lane = 0..ghost_lanes-1)
template <class T, int N>
__device__ __forceinline__ void ghost_face(T *u, const FaceItem &fi, int dir, bool bicubic,
                                           const GhostCubicTable<N> &tab, int lane) {
    constexpr int G = N + 2, NC = G * G, NB2 = N / 2, LN = ghost_lanes<N>();
    constexpr int64_t V = (int64_t)G * G * G;
    // A pass never reads a ghost cell of its own direction (sources are
    // planes interior along `dir`), so each lane issues all of its loads
    // before any of its stores: IT independent DRAM round trips in flight
    // instead of IT dependent ones.
    constexpr int IT = (NC + LN - 1) / LN;
    T *ud = u + (int64_t)fi.dst * V;
    const int xg = fi.lr == 0 ? -1 : N;
    T val[IT];
    if (fi.type == 0) {
        const T *us = u + (int64_t)fi.src * V;
        const int xs = fi.lr == 0 ? N - 1 : 0;
#pragma unroll
        for (int t = 0; t < IT; t++) {
            const int c = lane + LN * t;
            if (c >= NC) break;
            const int p = c % G - 1, q = c / G - 1;
            int is, js, ks;
            put3(dir, xs, p, q, is, js, ks);
            val[t] = us[cidx(G, is, js, ks)];
        }
#pragma unroll
        for (int t = 0; t < IT; t++) {
            const int c = lane + LN * t;
            if (c >= NC) break;
            const int p = c % G - 1, q = c / G - 1;
            int i, j, k;
            put3(dir, xg, p, q, i, j, k);
            ud[cidx(G, i, j, k)] = val[t];
        }
        return;
    }
    const T *uc = u + (int64_t)fi.src * V;
    const int xc = fi.lr == 0 ? N - 1 : 0;
    const int oa = fi.oa * NB2, ob = fi.ob * NB2;
    const int inner = fi.lr == 0 ? 1 : -1;
    auto B = [&](int pb, int qb) -> T {
        int ci, cj, ck;
        put3(dir, xc, pb + oa, qb + ob, ci, cj, ck);
        return uc[cidx(G, ci, cj, ck)];
    };
#pragma unroll
    for (int t = 0; t < IT; t++) {
        const int c = lane + LN * t;
        if (c >= NC) break;
        const int p = c % G - 1, q = c / G - 1;
        T uH;
        if (bicubic) {
            const int *cp = tab.c[p + 1], *cq = tab.c[q + 1];
            const double *wp = tab.w[p + 1], *wq = tab.w[q + 1];
            T bx[4];
#pragma unroll
            for (int m = 0; m < 4; m++)
                bx[m] = (T)wp[0] * B(cp[0], cq[m]) + (T)wp[1] * B(cp[1], cq[m]) + (T)wp[2] * B(cp[2], cq[m])
                      + (T)wp[3] * B(cp[3], cq[m]);
            uH = (T)wq[0] * bx[0] + (T)wq[1] * bx[1] + (T)wq[2] * bx[2] + (T)wq[3] * bx[3];
        } else {
            const int pc = fdiv2(p), qc = fdiv2(q);
            const int p1 = near_(p, pc), q1 = near_(q, qc);
            uH = ((T)9 * B(pc, qc) + B(p1, q1) + (T)3 * B(pc, q1) + (T)3 * B(p1, qc)) / (T)16;
        }
        int i0, j0, k0, iN, jN, kN;
        put3(dir, xg + inner, p, q, i0, j0, k0);
        put3(dir, xg + 2 * inner, p, q, iN, jN, kN);
        const T u0 = ud[cidx(G, i0, j0, k0)], uN = ud[cidx(G, iN, jN, kN)];
        val[t] = ((T)10 * u0 + (T)8 * uH - (T)3 * uN) / (T)15;
    }
#pragma unroll
    for (int t = 0; t < IT; t++) {
        const int c = lane + LN * t;
        if (c >= NC) break;
        const int p = c % G - 1, q = c / G - 1;
        int i, j, k;
        put3(dir, xg, p, q, i, j, k);
        ud[cidx(G, i, j, k)] = val[t];
    }
}

// Same-level faces (type 0, fmg_ghfix_samelev) as a flat copy: cell g of a
// list of type-0 items is ghost cell g % NC of face g / NC, at in-block
// offset (x+1) sd + (p+1) sa + (q+1) sb with the pass direction's strides.
// A thread serves K cells `stride` apart and issues its K item loads, then
// its K value loads, then its K stores: the gather is latency-bound, and
// HBM only fills with several round trips in flight per thread (K =
// ghost_k<N>(); fewer cells per thread measured slower, also on small
// passes, and K is a compile-time constant -- a run-time count measured
// slower).
constexpr int kGhostK = 4;
// from 8^3 blocks on (faces of >= 100 cells, passes of megabytes) eight
// cells per thread measured faster; below, four
template <int N>
__host__ __device__ constexpr int ghost_k() { return N >= 8 ? 8 : kGhostK; }
template <class T, int N>
__device__ __forceinline__ void ghost_copy(T *u, const FaceItem *items, int ncell, int dir, int g0, int stride) {
    constexpr int G = N + 2, NC = G * G, K = ghost_k<N>();
    constexpr int64_t V = (int64_t)G * G * G;
    const int sd = dir == 0 ? 1 : (dir == 1 ? G : G * G);
    const int sa = dir == 0 ? G : 1;
    const int sb = dir == 2 ? G : G * G;
    int64_t src[K], dst[K];
#pragma unroll
    for (int t = 0; t < K; t++) {
        const int g = g0 + t * stride;
        src[t] = -1;
        dst[t] = 0;
        if (g < ncell) {
            const int fidx = g / NC, c = g - fidx * NC;
            const FaceItem fi = items[fidx];
            const int base = (c % G) * sa + (c / G) * sb;
            const bool lo = fi.lr == 0;   // ghost plane x = -1 fed by the source's x = N-1, or N by 0
            dst[t] = (int64_t)fi.dst * V + base + (lo ? 0 : N + 1) * sd;
            src[t] = (int64_t)fi.src * V + base + (lo ? N : 1) * sd;
        }
    }
    T val[K];
#pragma unroll
    for (int t = 0; t < K; t++)
        if (src[t] >= 0) val[t] = u[src[t]];
#pragma unroll
    for (int t = 0; t < K; t++)
        if (src[t] >= 0) u[dst[t]] = val[t];
}

// Elements per copy unit of a same-level face in pass `dir`: the y pass
// copies rows of G contiguous values, the z pass planes of G^2 contiguous
// values, so both move whole 8- or 16-byte vectors -- the largest power of
// two up to 16 bytes that divides the row (y) or the plane (z).  Every
// block starts at a multiple of V = G^3 values and every row or plane at a
// multiple of G or G^2 values from it, so with a 16-byte aligned field (the
// host checks) each unit is aligned to its own size.  The x pass (one value
// per row) stays scalar.
template <class T, int N>
__host__ __device__ constexpr int ghost_vec(int dir) {
    constexpr int G = N + 2, CAP = 16 / (int)sizeof(T);
    const int len = dir == 1 ? G : (dir == 2 ? G * G : 1);
    int w = 1;
    while (2 * w <= CAP && len % (2 * w) == 0) w *= 2;
    return w;
}
template <class T, int W>
struct GhostVec;
template <class T>
struct GhostVec<T, 1> { using type = T; };
template <>
struct GhostVec<float, 2> { using type = float2; };
template <>
struct GhostVec<float, 4> { using type = float4; };
template <>
struct GhostVec<double, 2> { using type = double2; };
// the flat copy of ghost_copy in units of W values (W > 1: dir 1 or 2)
template <class T, int N, int W>
__device__ __forceinline__ void ghost_copy_vec(T *u, const FaceItem *items, int nunit, int dir, int g0, int stride) {
    using VT = typename GhostVec<T, W>::type;
    constexpr int G = N + 2, NU = G * G / W, K = ghost_k<N>();
    constexpr int64_t V = (int64_t)G * G * G;
    static_assert((G * G) % W == 0 && V % W == 0, "units stay inside a face and blocks stay aligned");
    const int sd = dir == 1 ? G : G * G;
    const int sb = dir == 2 ? G : G * G;
    int64_t src[K], dst[K];
#pragma unroll
    for (int t = 0; t < K; t++) {
        const int g = g0 + t * stride;
        src[t] = -1;
        dst[t] = 0;
        if (g < nunit) {
            const int fidx = g / NU, c = (g - fidx * NU) * W;
            const FaceItem fi = items[fidx];
            const int base = c % G + (c / G) * sb;
            const bool lo = fi.lr == 0;
            dst[t] = (int64_t)fi.dst * V + base + (lo ? 0 : N + 1) * sd;
            src[t] = (int64_t)fi.src * V + base + (lo ? N : 1) * sd;
        }
    }
    VT val[K];
#pragma unroll
    for (int t = 0; t < K; t++)
        if (src[t] >= 0) val[t] = *reinterpret_cast<const VT *>(u + src[t]);
#pragma unroll
    for (int t = 0; t < K; t++)
        if (src[t] >= 0) *reinterpret_cast<VT *>(u + dst[t]) = val[t];
}

// One ghost pass of (level, direction): the n0 same-level items0 by flat
// copy in the first CTAs (vectors of `vec` values: ghost_vec, or 1), the n1
// coarse-fine items1 (fmg_ghfix_parentlev) by ghost_face in the rest.  The
// two sets write disjoint ghost cells and read none of the pass direction,
// so they run side by side.
template <int N>
__host__ __device__ constexpr int ghost_copy_ctas(int n0, int vec = 1) {
    return (int)(((int64_t)n0 * ((N + 2) * (N + 2) / vec) + 256 * ghost_k<N>() - 1) / (256 * ghost_k<N>()));
}
// W: values per same-level copy unit (1, or ghost_vec<T, N>(dir) for a
// y or z pass on a 16-byte aligned field); one instantiation per width keeps
// the scalar x pass at its own register count
template <class T, int N, int W = 1>
__global__ void __launch_bounds__(256) k_ghost_faces(T *u, const FaceItem *__restrict__ items0, int n0,
                                                     const FaceItem *__restrict__ items1, int n1, int dir,
                                                     int cubic) {
    pdl_enter();
    constexpr int G = N + 2, NB2 = N / 2, LN = ghost_lanes<N>();
    const int nb0 = ghost_copy_ctas<N>(n0, W);
    if ((int)blockIdx.x < nb0) {
        const int g0 = (int)blockIdx.x * 256 * ghost_k<N>() + (int)threadIdx.x;
        if constexpr (W > 1)
            ghost_copy_vec<T, N, W>(u, items0, n0 * (G * G / W), dir, g0, 256);
        else
            ghost_copy<T, N>(u, items0, n0 * G * G, dir, g0, 256);
        return;
    }
    __shared__ GhostCubicTable<N> tab;
    const bool bicubic = cubic && NB2 + 2 >= 4;
    if (bicubic) {
        if (threadIdx.x < G) cubic_weights((int)threadIdx.x - 1, -1, NB2, tab.c[threadIdx.x], tab.w[threadIdx.x]);
        __syncthreads();
    }
    const int it = ((int)blockIdx.x - nb0) * (256 / LN) + (int)threadIdx.x / LN;
    if (it >= n1) return;
    ghost_face<T, N>(u, items1[it], dir, bicubic, tab, threadIdx.x % LN);
}

// ---------------------------------------------------------------------------
// one ghost fill of a whole AMR level in one launch
// ---------------------------------------------------------------------------
// fmg_ghostcell_fix fills a level by three passes, x then y then z
// (fmg_ghostcell.F90:49-54); pass d writes the d-ghost planes (whole
// transverse range) of the level's linked faces and reads no d-ghost plane.
// So the value a ghost cell ends with comes from the pass of its highest
// ghost dimension D whose face is filled, and that pass reads (a) cells
// interior along D of the same level -- which hold either interior values or
// ghost values of dimensions below D, themselves final after passes < D --
// and (b) coarse cells of the level above, complete before this level
// starts.  k_ghost_level writes those final values for a whole level in one
// launch.  Its work comes as host-built item lists (GItem), one list per
// kind of cell so that no warp mixes kinds:
//   - a face, edge or corner segment whose chain of passes runs through
//     same-level faces only ends up holding an interior cell of one block
//     (the neighbour across the highest ghost dimension, then its
//     neighbour across the next...): a flat copy;
//   - the face part of a coarse-fine face is the parentlev formula of its
//     coarse layer and two interior cells, as in ghost_face;
//   - the few edges and corners whose chain meets a coarse-fine or an
//     unfilled face follow the composition (ghost_value / ghost_pass_value,
//     depth <= 3).
// Every read is of an interior cell, a coarse cell or a ghost cell no pass
// of this fill writes; every write is a ghost cell of the level: no read
// meets a write of the same launch, and the same expressions as ghost_face /
// ghost_copy give bit-identical values.  A cell no pass writes is left
// alone.  Where the composition would read a ghost cell that a later pass of
// the same fill rewrites (possible next to the physical boundary, or when
// only one kind of face is filled), the host keeps the three passes for
// that level (Solver::ghost_merge_ok).
struct GFace {             // one face of one block for the level fills
    int32_t src;           // same-level neighbour, parent-level neighbour, or -1
    int8_t type;           // 0 same level, 1 coarse-fine, 2 physical boundary
    int8_t pad[3];
};
// true when a fill of kind `sel` (-1 both kinds, 0 same level only, 1
// coarse-fine only) writes the ghost plane of a face of this type
__host__ __device__ __forceinline__ bool gface_filled(int type, int sel) {
    return (type == 0 && sel != 1) || (type == 1 && sel != 0);
}

template <class T, int N>
struct GhostLevelArgs {
    const T *u; const GFace *gf; const int8_t *oct; int sel; bool bicubic;
    const GhostCubicTable<N> *tab;
};

template <class T, int N, int D>
__device__ __noinline__ T ghost_pass_value(const GhostLevelArgs<T, N> &a, GFace f, int lr, int X, int i, int j, int k);

// state of cell (i,j,k) of block X after passes 0..DL of the fill; the
// coordinates of dimensions above DL are interior.  Not inlined: one copy
// of each depth keeps the code small (inlined, the three-deep composition
// multiplied the interpolation code and the kernel ran from instruction
// cache misses on levels with many coarse-fine faces).
template <class T, int N, int DL>
__device__ __noinline__ T ghost_value(const GhostLevelArgs<T, N> &a, int X, int i, int j, int k) {
    constexpr int G = N + 2;
    constexpr int64_t V = (int64_t)G * G * G;
    if constexpr (DL >= 0) {
        const int c = DL == 0 ? i : (DL == 1 ? j : k);
        if (c == -1 || c == N) {
            const int lr = c == N ? 1 : 0;
            const GFace f = a.gf[6 * X + lr + 2 * DL];
            if (gface_filled(f.type, a.sel)) return ghost_pass_value<T, N, DL>(a, f, lr, X, i, j, k);
        }
        return ghost_value<T, N, DL - 1>(a, X, i, j, k);
    } else {
        return a.u[(int64_t)X * V + cidx(G, i, j, k)];
    }
}

// the value pass D writes into cell (i,j,k) (on the D-ghost plane of side lr)
template <class T, int N, int D>
__device__ __noinline__ T ghost_pass_value(const GhostLevelArgs<T, N> &a, GFace f, int lr, int X, int i, int j, int k) {
    constexpr int G = N + 2, NB2 = N / 2;
    constexpr int64_t V = (int64_t)G * G * G;
    if (f.type == 0) {   // fmg_ghfix_samelev: the neighbour's cell on the opposite boundary plane
        const int xs = lr == 0 ? N - 1 : 0;
        return ghost_value<T, N, D - 1>(a, f.src, D == 0 ? xs : i, D == 1 ? xs : j, D == 2 ? xs : k);
    }
    // fmg_ghfix_parentlev: transverse interpolation of the coarse layer, then
    // the quadratic normal formula with the two inner fine cells
    const int p = D == 0 ? j : i, q = D == 2 ? j : k;
    const T *uc = a.u + (int64_t)f.src * V;
    const int xc = lr == 0 ? N - 1 : 0;
    const int oa = a.oct[3 * X + tra(D)] * NB2, ob = a.oct[3 * X + trb(D)] * NB2;
    auto B = [&](int pb, int qb) -> T {
        int ci, cj, ck;
        put3(D, xc, pb + oa, qb + ob, ci, cj, ck);
        return uc[cidx(G, ci, cj, ck)];
    };
    T uH;
    if (a.bicubic) {
        const int *cp = a.tab->c[p + 1], *cq = a.tab->c[q + 1];
        const double *wp = a.tab->w[p + 1], *wq = a.tab->w[q + 1];
        T bx[4];
#pragma unroll
        for (int m = 0; m < 4; m++)
            bx[m] = (T)wp[0] * B(cp[0], cq[m]) + (T)wp[1] * B(cp[1], cq[m]) + (T)wp[2] * B(cp[2], cq[m])
                  + (T)wp[3] * B(cp[3], cq[m]);
        uH = (T)wq[0] * bx[0] + (T)wq[1] * bx[1] + (T)wq[2] * bx[2] + (T)wq[3] * bx[3];
    } else {
        const int pc = fdiv2(p), qc = fdiv2(q);
        const int p1 = near_(p, pc), q1 = near_(q, qc);
        uH = ((T)9 * B(pc, qc) + B(p1, q1) + (T)3 * B(pc, q1) + (T)3 * B(p1, qc)) / (T)16;
    }
    const int xg = lr == 0 ? -1 : N, inner = lr == 0 ? 1 : -1;
    const int x0 = xg + inner, xN = xg + 2 * inner;
    const T u0 = ghost_value<T, N, D - 1>(a, X, D == 0 ? x0 : i, D == 1 ? x0 : j, D == 2 ? x0 : k);
    const T uN = ghost_value<T, N, D - 1>(a, X, D == 0 ? xN : i, D == 1 ? xN : j, D == 2 ? xN : k);
    return ((T)10 * u0 + (T)8 * uH - (T)3 * uN) / (T)15;
}

// the final value of shell cell (i,j,k) of block X, or false when no pass of
// the fill writes it (general composition, for cells whose chain meets a
// coarse-fine or an unfilled face)
template <class T, int N>
__device__ __noinline__ bool ghost_cell_general(const GhostLevelArgs<T, N> &a, int X, int i, int j, int k, T &out) {
    const int cs[3] = {i, j, k};
#pragma unroll
    for (int d = 2; d >= 0; d--) {
        if (cs[d] != -1 && cs[d] != N) continue;
        const int lr = cs[d] == N ? 1 : 0;
        const GFace f = a.gf[6 * X + lr + 2 * d];
        if (!gface_filled(f.type, a.sel)) continue;
        out = d == 2 ? ghost_pass_value<T, N, 2>(a, f, lr, X, i, j, k)
                     : (d == 1 ? ghost_pass_value<T, N, 1>(a, f, lr, X, i, j, k)
                               : ghost_pass_value<T, N, 0>(a, f, lr, X, i, j, k));
        return true;
    }
    return false;
}

// shell segment of a cell: 3^3 pattern of (low ghost, interior, high ghost)
// per dimension, (sx+1) + 3 (sy+1) + 9 (sz+1), the interior 13 excluded:
// entries 0..12 and 14..26 map to 0..25
__host__ __device__ __forceinline__ int shell_segment(int sx, int sy, int sz) {
    const int s = (sx + 1) + 3 * (sy + 1) + 9 * (sz + 1);
    return s < 13 ? s : s - 1;
}
__host__ __device__ __forceinline__ void segment_sides(int seg, int &sx, int &sy, int &sz) {
    const int s = seg < 13 ? seg : seg + 1;
    sx = s % 3 - 1;
    sy = (s / 3) % 3 - 1;
    sz = s / 9 - 1;
}

// Kind of a shell segment of a block in one level fill (kind26[26 X + seg]):
//   >= 0  the chain of the passes runs through filled same-level faces only
//         and the segment ends up holding interior cells of that block (the
//         neighbour across the highest ghost dimension, then its neighbour
//         across the next...), at the cell's coordinates wrapped into it;
//   -1    no pass of the fill writes the segment;
//   -2    a filled coarse-fine face (face segment): the parentlev formula;
//   -3    anything else (edges and corners whose chain meets a coarse-fine
//         or an unfilled face): the general composition, done by the
//         trailing CTAs of the launch from a list of (block, segment) items.
constexpr int kSegSkip = -1, kSegCF = -2, kSegGeneral = -3;
struct GItem {
    int32_t dst;
    int8_t seg, pad[3];
};

// shell cells of one block, grouped by the highest ghost dimension (the
// pass that writes them last): 2 N^2 on x planes, 2 (N+2) N on y planes,
// 2 (N+2)^2 on z planes -- every cell once, all of a block's together
template <int N>
__host__ __device__ constexpr int ghost_shell() { return 2 * (N * N + (N + 2) * N + (N + 2) * (N + 2)); }

// cell r (0 .. ghost_shell - 1) of a block's shell
template <int N>
__device__ __forceinline__ void shell_cell(int r0, int &i, int &j, int &k) {
    constexpr int A0 = N * N, A1 = (N + 2) * N, A2 = (N + 2) * (N + 2);
    if (r0 < 2 * A0) {
        const int side = r0 / A0, t0 = r0 - side * A0;
        i = side ? N : -1; j = t0 % N; k = t0 / N;
    } else if (r0 < 2 * A0 + 2 * A1) {
        const int r = r0 - 2 * A0, side = r / A1, t1 = r - side * A1;
        i = t1 % (N + 2) - 1; j = side ? N : -1; k = t1 / (N + 2);
    } else {
        const int r = r0 - 2 * A0 - 2 * A1, side = r / A2, t2 = r - side * A2;
        i = t2 % (N + 2) - 1; j = t2 / (N + 2) - 1; k = side ? N : -1;
    }
}

// the parentlev value of cell (i,j,k) on the face part (transverse interior)
// of coarse-fine face (D, lr) of block X, coarse block C (as ghost_face)
template <class T, int N>
__device__ __noinline__ T ghost_cf_face(const T *u, const int8_t *oct, int X, int C, int D, int lr, int i, int j, int k,
                                        bool bicubic, const GhostCubicTable<N> *tab) {
    constexpr int G = N + 2, NB2 = N / 2;
    constexpr int64_t V = (int64_t)G * G * G;
    const int p = D == 0 ? j : i, q = D == 2 ? j : k;
    const T *uc = u + (int64_t)C * V;
    const T *ud = u + (int64_t)X * V;
    const int xc = lr == 0 ? N - 1 : 0;
    const int oa = oct[3 * X + tra(D)] * NB2, ob = oct[3 * X + trb(D)] * NB2;
    auto B = [&](int pb, int qb) -> T {
        int ci, cj, ck;
        put3(D, xc, pb + oa, qb + ob, ci, cj, ck);
        return uc[cidx(G, ci, cj, ck)];
    };
    T uH;
    if (bicubic) {
        const int *cp = tab->c[p + 1], *cq = tab->c[q + 1];
        const double *wp = tab->w[p + 1], *wq = tab->w[q + 1];
        T bx[4];
#pragma unroll
        for (int m = 0; m < 4; m++)
            bx[m] = (T)wp[0] * B(cp[0], cq[m]) + (T)wp[1] * B(cp[1], cq[m]) + (T)wp[2] * B(cp[2], cq[m])
                  + (T)wp[3] * B(cp[3], cq[m]);
        uH = (T)wq[0] * bx[0] + (T)wq[1] * bx[1] + (T)wq[2] * bx[2] + (T)wq[3] * bx[3];
    } else {
        const int pc = fdiv2(p), qc = fdiv2(q);
        const int p1 = near_(p, pc), q1 = near_(q, qc);
        uH = ((T)9 * B(pc, qc) + B(p1, q1) + (T)3 * B(pc, q1) + (T)3 * B(p1, qc)) / (T)16;
    }
    const int xg = lr ? N : -1, inner = lr ? -1 : 1;
    int i0, j0, k0, iN, jN, kN;
    put3(D, xg + inner, p, q, i0, j0, k0);
    put3(D, xg + 2 * inner, p, q, iN, jN, kN);
    const T u0 = ud[cidx(G, i0, j0, k0)], uN = ud[cidx(G, iN, jN, kN)];
    return ((T)10 * u0 + (T)8 * uH - (T)3 * uN) / (T)15;
}

// One fill of the level's blocks first .. first+nblk-1.  The first `sweep`
// CTAs give each warp one block: the block's 26 segment kinds go to shared
// memory, and the warp walks the block's shell through a per-CTA table of
// (destination offset, wrapped source offset, segment) for every shell
// cell, so a copied cell costs two shared loads, one load and one store
// (decoding the cell from a flat index each time measured issue-bound).
// The remaining CTAs take the general items.
constexpr int kGhostWarps = 8;   // blocks per sweep CTA (one per warp)
template <int N>
__host__ __device__ constexpr int ghost_sweep_ctas(int nblk) { return (nblk + kGhostWarps - 1) / kGhostWarps; }
template <int N>
__host__ __device__ constexpr int ghost_general_ctas(int items) {
    return (int)(((int64_t)items * N + 255) / 256);   // N cells per item (corners use the first)
}
template <int N>
struct ShellTable {
    uint32_t off[ghost_shell<N>()];   // in-block offset of the cell | wrapped offset << 16 (G^3 < 2^16)
    uint8_t seg[ghost_shell<N>()];
};

template <class T, int N>
__global__ void __launch_bounds__(256) k_ghost_level(T *u, const int32_t *__restrict__ kind26,
                                                     const GItem *__restrict__ gen, int ngen, int first, int nblk,
                                                     int sweep, const GFace *__restrict__ gf,
                                                     const int8_t *__restrict__ oct, int sel, int cubic) {
    pdl_enter();
    constexpr int G = N + 2, NB2 = N / 2, SH = ghost_shell<N>(), U = 4;
    constexpr int64_t V = (int64_t)G * G * G;
    static_assert(G * G * G < 65536, "offsets fit 16 bits");
    __shared__ GhostCubicTable<N> tab;
    const bool bicubic = cubic && NB2 + 2 >= 4 && sel != 0;
    if (bicubic) {   // launch-uniform
        if (threadIdx.x < G) cubic_weights((int)threadIdx.x - 1, -1, NB2, tab.c[threadIdx.x], tab.w[threadIdx.x]);
        __syncthreads();
    }
    if ((int)blockIdx.x < sweep) {
        __shared__ ShellTable<N> st;
        __shared__ int wk[kGhostWarps][26];
        for (int r = threadIdx.x; r < SH; r += blockDim.x) {
            int i, j, k;
            shell_cell<N>(r, i, j, k);
            auto wrap = [](int x) { return x < 0 ? N - 1 : (x >= N ? 0 : x); };
            st.off[r] = (uint32_t)cidx(G, i, j, k) | ((uint32_t)cidx(G, wrap(i), wrap(j), wrap(k)) << 16);
            const int sx = i < 0 ? -1 : (i >= N ? 1 : 0), sy = j < 0 ? -1 : (j >= N ? 1 : 0),
                      sz = k < 0 ? -1 : (k >= N ? 1 : 0);
            st.seg[r] = (uint8_t)shell_segment(sx, sy, sz);
        }
        __syncthreads();
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int bq = (int)blockIdx.x * kGhostWarps + w;
        if (bq >= nblk) return;
        const int X = first + bq;
        if (lane < 26) wk[w][lane] = kind26[26 * (int64_t)X + lane];
        __syncwarp();
        T *ud = u + (int64_t)X * V;
        for (int r0 = 0; r0 < SH; r0 += 32 * U) {
            T val[U];
            int dof[U];
#pragma unroll
            for (int q = 0; q < U; q++) {
                const int r = r0 + q * 32 + lane;
                dof[q] = -1;
                if (r >= SH) continue;
                const uint32_t o = st.off[r];
                const int kd = wk[w][st.seg[r]];
                if (kd >= 0) {
                    val[q] = u[(int64_t)kd * V + (o >> 16)];
                    dof[q] = (int)(o & 0xffffu);
                } else if (kd == kSegCF) {
                    const int c = (int)(o & 0xffffu);
                    const int i = c % G - 1, j = (c / G) % G - 1, k = c / (G * G) - 1;
                    const int D = (i == -1 || i == N) ? 0 : ((j == -1 || j == N) ? 1 : 2);
                    const int cc = D == 0 ? i : (D == 1 ? j : k);
                    const int lr = cc == N ? 1 : 0;
                    val[q] = ghost_cf_face<T, N>(u, oct, X, gf[6 * X + lr + 2 * D].src, D, lr, i, j, k, bicubic, &tab);
                    dof[q] = c;
                }
            }
#pragma unroll
            for (int q = 0; q < U; q++)
                if (dof[q] >= 0) ud[dof[q]] = val[q];
        }
        return;
    }
    // general items: N cells per item (the free coordinate of an edge; a
    // corner uses cell 0 only); loads happen in the composition, then one store
    const int64_t g = (int64_t)((int)blockIdx.x - sweep) * 256 + threadIdx.x;
    const int q = (int)(g / N), c = (int)(g - (int64_t)q * N);
    if (q >= ngen) return;
    const GItem e = gen[q];
    int sx, sy, sz;
    segment_sides(e.seg, sx, sy, sz);
    if (sx && sy && sz && c != 0) return;
    const int sd[3] = {sx, sy, sz};
    int o[3];
#pragma unroll
    for (int d = 0; d < 3; d++) o[d] = sd[d] < 0 ? -1 : (sd[d] > 0 ? N : c);
    const GhostLevelArgs<T, N> a{u, gf, oct, sel, bicubic, &tab};
    T v;
    if (ghost_cell_general<T, N>(a, e.dst, o[0], o[1], o[2], v)) u[(int64_t)e.dst * V + cidx(G, o[0], o[1], o[2])] = v;
}

// ---------------------------------------------------------------------------
// staging of BPC consecutive listed blocks (G^3 each) into shared memory
// ---------------------------------------------------------------------------
template <int N>
struct Tile {
    static constexpr int G = N + 2;
    static constexpr int V = G * G * G;
    static constexpr int CELLS = N * N * N;
    // blocks per CTA: a CTA covers at least 512 cells
    static constexpr int BPC = CELLS >= 512 ? 1 : 512 / CELLS;
};

template <class T, int N, int BPCX = Tile<N>::BPC>
__device__ __forceinline__ void stage_blocks(T *sh, const T *u, const int32_t *__restrict__ blocks,
                                             int first, int nblk) {
    using Tl = Tile<N>;
    for (int t = threadIdx.x; t < BPCX * Tl::V; t += blockDim.x) {
        const int q = t / Tl::V, r = t - q * Tl::V;
        if (first + q < nblk) sh[t] = u[(int64_t)blocks[first + q] * Tl::V + r];
    }
}

// flux / divergence on a staged tile, with the reflux substitution of
// Flux<T> (sfm_device.cuh) for coarse faces covered by finer blocks
template <class T, int N>
struct TileFlux {
    const T *ub; T hi; const int *slot; const double *rbuf;
    __device__ __forceinline__ T f(int dir, int i, int j, int k) const {
        constexpr int G = N + 2;
        if (slot) {
            const int x = dir == 0 ? i : (dir == 1 ? j : k);
            if (x == N - 1 || x == -1) {
                const int s = slot[(x == -1 ? 0 : 1) + 2 * dir];
                if (s >= 0) {
                    const int a = dir == 0 ? j : i, c = dir == 2 ? j : k;
                    return (T)rbuf[(int64_t)s * N * N + (int64_t)c * N + a];
                }
            }
        }
        const int i1 = i + (dir == 0), j1 = j + (dir == 1), k1 = k + (dir == 2);
        return (ub[cidx(G, i1, j1, k1)] - ub[cidx(G, i, j, k)]) * hi;
    }
    __device__ __forceinline__ T div(int i, int j, int k) const {
        T t = f(0, i, j, k) - f(0, i - 1, j, k);
        t = t + f(1, i, j, k);
        t = t - f(1, i, j - 1, k);
        t = t + f(2, i, j, k);
        t = t - f(2, i, j, k - 1);
        return t;
    }
};

// ---------------------------------------------------------------------------
// red-black colour sweep on listed blocks (fmg_poisson_relax / vmg_poisson_relax)
// ---------------------------------------------------------------------------
// CTA-wide max of non-negative doubles, folded into *out with one atomic
__device__ __forceinline__ void cta_max_atomic(double m, unsigned long long *out) {
    __shared__ double wm[32];
    for (int o = 16; o > 0; o >>= 1) {
        const double t2 = __shfl_xor_sync(0xffffffffu, m, o);
        m = t2 > m ? t2 : m;
    }
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) r = wm[w] > r ? wm[w] : r;
        if (r > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(r));
    }
}

// shared buffers of one CTA's tiled colour sweep
template <class T, int N>
struct RelaxTileSmem {
    T sh[Tile<N>::BPC * Tile<N>::V];
    int ssl[Tile<N>::BPC][6];
    T shh[Tile<N>::BPC], shi[Tile<N>::BPC];
};

// one colour (ipass 1 or 2), or sw > 0 full sweeps (a mixed-schedule
// choice), over tiles tile0, tile0 + tstride, ... of BPC consecutive listed
// blocks: each block with its ghost shell staged in shared memory, updated,
// interior rows written back; |resh2| folded into m.
template <class T, int N>
__device__ __forceinline__ void relax_tiles(RelaxTileSmem<T, N> &sm, T *u, const T *__restrict__ rhs,
                                            const int32_t *__restrict__ blocks, int nblk,
                                            const double *__restrict__ h0, const int32_t *__restrict__ level,
                                            const int32_t *__restrict__ rslot, const double *rbuf,
                                            int f, int ipass, int sw, int tile0, int tstride, double &m) {
    using Tl = Tile<N>;
    constexpr int G = Tl::G, V = Tl::V, BPC = Tl::BPC, HALF = Tl::CELLS / 2;
    const int ntiles = (nblk + BPC - 1) / BPC;
    for (int tile = tile0; tile < ntiles; tile += tstride) {
        const int first = tile * BPC;
        stage_blocks<T, N>(sm.sh, u, blocks, first, nblk);
        if (threadIdx.x < BPC * 6) {
            const int q = threadIdx.x / 6, fc = threadIdx.x % 6;
            sm.ssl[q][fc] = (rslot && first + q < nblk) ? rslot[6 * blocks[first + q] + fc] : -1;
        }
        if (threadIdx.x < BPC && first + (int)threadIdx.x < nblk) {
            const double hd = hlev(h0, level[blocks[first + threadIdx.x]], f);
            sm.shh[threadIdx.x] = (T)hd;
            sm.shi[threadIdx.x] = (T)(1.0 / hd);
        }
        __syncthreads();
        // sw > 0: sw full sweeps, each colour reading the previous one's new
        // values from the stage (ghost cells and reflux fluxes as staged)
        for (int q2 = 0; q2 < (sw > 0 ? 2 * sw : 1); q2++) {
            const int pass = sw > 0 ? 1 + (q2 & 1) : ipass;
            for (int t = threadIdx.x; t < BPC * HALF; t += blockDim.x) {
                const int q = t / HALF, r = t - q * HALF;
                if (first + q >= nblk) continue;
                const int b = blocks[first + q];
                constexpr int HN = N / 2;
                const int i2 = r % HN, j = (r / HN) % N, k = r / (HN * N);
                const int i = 2 * i2 + ((j + k + pass) & 1);
                const T hh = sm.shh[q], hi = sm.shi[q];
                T *ub = sm.sh + q * V;
                TileFlux<T, N> F{ub, hi, rslot ? sm.ssl[q] : nullptr, rbuf};
                const int c = (int)cidx(G, i, j, k);
                const T resh2 = (F.div(i, j, k) - rhs[(int64_t)b * V + c] * hh) * hh;
                ub[c] = ub[c] + (T)(1.0 / 6.0) * resh2;   // only this thread reads this cell
                const double a = fabs((double)resh2);
                m = a > m ? a : m;
            }
            __syncthreads();
        }
        // write back the interior rows of every staged block
        for (int t = threadIdx.x; t < BPC * Tl::CELLS; t += blockDim.x) {
            const int q = t / Tl::CELLS, r = t - q * Tl::CELLS;
            if (first + q >= nblk) continue;
            const int i = r % N, j = (r / N) % N, k = r / (N * N);
            const int c = (int)cidx(G, i, j, k);
            u[(int64_t)blocks[first + q] * V + c] = sm.sh[q * V + c];
        }
        __syncthreads();
    }
}

// persistent: each CTA walks tiles of BPC consecutive listed blocks
template <class T, int N>
__global__ void __launch_bounds__(256) k_relax_tiled(T *__restrict__ u, const T *__restrict__ rhs,
                                                     const int32_t *__restrict__ blocks, int nblk,
                                                     const double *__restrict__ h0, const int32_t *__restrict__ level,
                                                     const int32_t *__restrict__ rslot, const double *__restrict__ rbuf,
                                                     int f, int ipass, int sw, unsigned long long *out) {
    pdl_enter();
    __shared__ RelaxTileSmem<T, N> sm;
    double m = 0.0;
    relax_tiles<T, N>(sm, u, rhs, blocks, nblk, h0, level, rslot, rbuf, f, ipass, sw, blockIdx.x, gridDim.x, m);
    cta_max_atomic(m, out);
}

// ---------------------------------------------------------------------------
// bulk-copy pipeline (1D cp.async.bulk, no multicast) for the block sweeps
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: false after `limit` unsuccessful polls
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t limit) {
    for (uint32_t t = 0; t < limit; t++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// bounded wait that also gives up as soon as *abort is set
__device__ __forceinline__ bool mbar_wait_bounded_abort(uint64_t *bar, uint32_t parity, uint32_t limit,
                                                        const int *abort) {
    for (uint32_t t = 0; t < limit; t++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*(const volatile int *)abort) return false;
    }
    return false;
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void bulk_store(void *dst, const void *src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

constexpr uint32_t kWaitPolls = 1u << 20;   // bound on every mbarrier wait of a sweep

// stages of the bulk pipeline: up to 3 within 48 KB of u + rhs tiles (3
// stages keep 8 CTAs per SM; deeper rings measured slower: 4 -> 11%, 6 -> 36%).
// [LO, LO + SPAN) is the 16-byte-aligned element range of a block that
// holds every interior cell (cidx of (0,0,0) to (N-1,N-1,N-1)).
template <class T, int N>
struct BulkPlan {
    static constexpr int G = N + 2, V = G * G * G;
    static constexpr int STAGE_BYTES = 2 * Tile<N>::BPC * V * (int)sizeof(T);
    static constexpr int S0 = 49152 / STAGE_BYTES;
    static constexpr int S = S0 >= 3 ? 3 : (S0 >= 2 ? S0 : 2);
    static constexpr int SMEM = S * STAGE_BYTES;
    static constexpr int EPB = 16 / (int)sizeof(T);
    static constexpr int LO = (1 + G + G * G) / EPB * EPB;
    static constexpr int HI = ((N + N * G + N * G * G) + 1 + EPB - 1) / EPB * EPB;
    static constexpr int SPAN = HI - LO;
    static_assert(HI <= V && (V * (int)sizeof(T)) % 16 == 0, "span within the block, blocks 16-byte aligned");
};

// barrier `id` of `nthreads` threads (a multiple of 32, whole warps) that
// also ORs a predicate over them: every participant gets the same result
__device__ __forceinline__ bool consumers_sync_or(int id, int nthreads, bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, %2, %3, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Red-black colour sweep, warp-specialised.  Warp 0 produces: for each tile
// it waits until the consumers have released a stage (mbarrier `empty`),
// loads the tile's per-block data (block ids, reflux slots, cell widths) into
// that stage and brings the whole u blocks (ghost shell included) and the
// interior span of rhs with 1D bulk async copies (mbarrier `full`).  Warps
// 1..7 consume: each warp computes its cells of one colour from the staged
// block (the arithmetic of k_relax_tiled), stores the new values straight to
// u and releases the stage -- so a stage can be refilled as soon as it has
// been read, and the producer's latencies stay off the consumers' path.
// Every mbarrier wait is bounded: a wait that gives up sets *err, the warp
// leaves, and the producer stops issuing.  The consumers' wait for a stage
// polls at most `cpolls` times (kWaitPolls in a solve; a test sets it to 0
// to make every such wait give up and check the error path); the
// producer's wait for a free stage gives up at kWaitPolls or as soon as a
// consumer has given up; the final drain of copies still in flight always
// polls up to kWaitPolls, so no bulk copy writes shared memory after the
// CTA exits.  Every give-up decision is made warp-uniform (vote), so no
// lane waits at a warp barrier for a lane that has left.
// resident CTAs per SM the bulk ring's shared memory allows: the register
// budget that leaves (at 4^3 blocks ptxas otherwise settles on 32 registers
// and spills)
template <class T, int N, int NT = 256>
__host__ __device__ constexpr int relax_bulk_min_ctas() {
    // bounded by the ring's shared memory, 8, and the 2048 threads of an SM
    return (228 * 1024) / (BulkPlan<T, N>::SMEM + 1024) < (2048 / NT < 8 ? 2048 / NT : 8)
               ? (228 * 1024) / (BulkPlan<T, N>::SMEM + 1024)
               : (2048 / NT < 8 ? 2048 / NT : 8);
}
// threads of k_relax_bulk: warp 0 produces, the others consume.  A 16^3
// block's stages allow only one or two CTAs per SM, so those CTAs get 15
// consumer warps instead of 7.
// (the default; the autotuner may choose the other count per block edge)
template <int N>
__host__ __device__ constexpr int relax_bulk_threads() { return N >= 16 ? 512 : 256; }
//
// SW > 0 (a choice of the mixed path's schedule, never of the FP64 path):
// SW full red-black sweeps of every staged block in one pass -- each
// colour's new values go back into the stage, the consumer warps meet at a
// named barrier, and the next colour reads them there, with the block's
// ghost cells and reflux fluxes as they were before the launch (the
// reference refreshes them between the colours, fmg_poisson.F90:160-165);
// only the last sweep's values are stored to u.  u and rhs are read once
// and u written once per launch.  A consumer warp whose stage wait failed
// skips the first colour and still reaches the tile's first barrier, which
// ORs the failures: every consumer warp leaves after it, so none waits at a
// barrier for one that has gone.  SW = 0: the one colour `ipass`.
template <class T, int N, int NT = relax_bulk_threads<N>(), int SW = 0>
__global__ void __launch_bounds__(NT, relax_bulk_min_ctas<T, N, NT>())
    k_relax_bulk(T *__restrict__ u, const T *__restrict__ rhs,
                                                    const int32_t *__restrict__ blocks, int nblk,
                                                    const double *__restrict__ h0, const int32_t *__restrict__ level,
                                                    const int32_t *__restrict__ rslot, const double *__restrict__ rbuf,
                                                    int f, int ipass, unsigned long long *out, int *err,
                                                    uint32_t cpolls) {
    pdl_enter();
    using Tl = Tile<N>;
    using Pl = BulkPlan<T, N>;
    constexpr int G = Tl::G, V = Tl::V, BPC = Tl::BPC, HALF = Tl::CELLS / 2, S = Pl::S;
    constexpr int NCW = NT / 32 - 1, NCT = 32 * NCW;   // consumer warps / threads
    constexpr uint32_t BB = (uint32_t)(V * sizeof(T));
    constexpr int LO = Pl::LO;
    constexpr uint32_t SB = (uint32_t)(Pl::SPAN * sizeof(T));
    static_assert(BB % 16 == 0 && SB % 16 == 0 && (LO * sizeof(T)) % 16 == 0, "bulk copies move 16-byte units");
    extern __shared__ __align__(128) unsigned char bulk_smem[];
    T *ust = reinterpret_cast<T *>(bulk_smem);   // [S][BPC][V]
    T *rst = ust + S * BPC * V;                  // [S][BPC][V]
    __shared__ __align__(8) uint64_t full[S], empty[S];
    // pab: the producer gave up; cab: a consumer warp gave up
    __shared__ int issued[S], consumed[S], pab, cab;
    // per-block data of the tiles, by this CTA's step index: a ring of two
    // windows of R steps; the producer fills a whole window at once (one
    // latency for R tiles) S steps into the previous window, when every
    // consumer (at most S steps behind) has left the window it overwrites
    constexpr int R = (32 / BPC) > 2 * S ? 32 / BPC : 2 * S;
    __shared__ int bid[2 * R][BPC];
    __shared__ int ssl[2 * R][BPC][6];
    __shared__ int8_t hasr[2 * R][BPC];   // a face of the block takes a reflux flux
    __shared__ T shh[2 * R][BPC], shi[2 * R][BPC];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ntiles = (nblk + BPC - 1) / BPC;
    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NCW);
            issued[s] = 0;
            consumed[s] = 0;
        }
        pab = 0;
        cab = 0;
        mbar_init_fence();
    }
    __syncthreads();
    double m = 0.0;
    const int nsteps = ntiles > (int)blockIdx.x ? (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
    auto fill_window = [&](int w) {   // warp 0
        for (int e = lane; e < R * BPC; e += 32) {
            const int step = w * R + e / BPC, q = e % BPC, slot = step % (2 * R);
            const int first = ((int)blockIdx.x + step * (int)gridDim.x) * BPC;
            if (step < nsteps && first + q < nblk) {
                const int b = blocks[first + q];
                bid[slot][q] = b;
                int any = 0;
                for (int fc = 0; fc < 6; fc++) {
                    const int v = rslot ? rslot[6 * b + fc] : -1;
                    ssl[slot][q][fc] = v;
                    any |= v >= 0;
                }
                hasr[slot][q] = (int8_t)any;
                const double hd = hlev(h0, level[b], f);
                shh[slot][q] = (T)hd;
                shi[slot][q] = (T)(1.0 / hd);
            } else {
                for (int fc = 0; fc < 6; fc++) ssl[slot][q][fc] = -1;
                hasr[slot][q] = 0;
            }
        }
        __syncwarp();
    };
    if (warp == 0) {
        fill_window(0);
        int it = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
            const int s = it % S;
            if (it >= S) {
                const bool ok =
                    __all_sync(0xffffffffu, mbar_wait_bounded_abort(&empty[s], (uint32_t)((it / S - 1) & 1), kWaitPolls, &cab));
                if (!ok) {
                    if (lane == 0) pab = 1;
                    break;
                }
            }
            if (__any_sync(0xffffffffu, *(volatile int *)&cab)) break;
            if (it % R == S && (it / R + 1) * R < nsteps) fill_window(it / R + 1);
            const int first = tile * BPC;
            const int cnt = nblk - first < BPC ? nblk - first : BPC;
            const int slot = it % (2 * R);
            if (lane == 0) {
                issued[s]++;
                mbar_expect_tx(&full[s], (uint32_t)cnt * (BB + SB));   // releases the per-block data
            }
            __syncwarp();
            for (int q = lane; q < cnt; q += 32) {
                const int64_t b = bid[slot][q];
                bulk_load(ust + (s * BPC + q) * V, u + b * V, BB, &full[s]);
                bulk_load(rst + (s * BPC + q) * V + LO, rhs + b * V + LO, SB, &full[s]);
            }
        }
    } else {
        // Cells of one colour depend only on cells of the other colour, so
        // each consumer thread stores its updated cells straight to u and no
        // consumer waits for another: a warp waits for the stage, updates,
        // stores and releases the stage on its own.
        const int ct = tid - 32;   // consumer thread 0..NCT-1
        T mt = (T)0;               // max |resh2| (exact in T; widened once)
        int it = 0;
        // fused sweeps: cell t = ct + x NCT of each tile's colour-1 cells
        // (and its x neighbour, the colour-2 cell of t) for x < ITER
        constexpr int ITER = SW > 0 ? (BPC * HALF + NCT - 1) / NCT : 1;
        // block, in-block coordinates of the colour-1 cell and the step to
        // its x neighbour
        auto cell_of = [&](int x, int &q, int &i1, int &j, int &k, int &d1) {
            const int t = ct + x * NCT;
            q = t / HALF;
            const int r = t - q * HALF;
            constexpr int HN = N / 2;
            const int i2 = r % HN;
            j = (r / HN) % N;
            k = r / (HN * N);
            const int p1 = (j + k + 1) & 1;
            i1 = 2 * i2 + p1;
            d1 = 1 - 2 * p1;
        };
        // (recomputed where used: held across the tile loop they cost
        // registers the 7-CTA occupancy does not have)
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
            const int s = it % S;
            const bool got = __all_sync(0xffffffffu, mbar_wait_bounded(&full[s], (uint32_t)((it / S) & 1), cpolls));
            if constexpr (SW == 0) {
                if (!got) {
                    if (lane == 0) atomicExch(&cab, 1);
                    break;
                }
            }
            const int first = tile * BPC;
            const int slot = it % (2 * R);
            T *ut = ust + s * BPC * V;
            const T *rt = rst + s * BPC * V;
            // keep: the new values go back into the stage for a later colour;
            // store: they go to u
            auto colour = [&](int pass, bool keep, bool store) {
                for (int t = ct; t < BPC * HALF; t += NCT) {
                    const int q = t / HALF, r = t - q * HALF;
                    if (first + q >= nblk) continue;
                    constexpr int HN = N / 2;
                    const int i2 = r % HN, j = (r / HN) % N, k = r / (HN * N);
                    const int i = 2 * i2 + ((j + k + pass) & 1);
                    const T hh = shh[slot][q], hi = shi[slot][q];
                    T *ub = ut + q * V;
                    // blocks without a reflux face (a warp's cells share a block)
                    // skip the per-face slot tests: same fluxes, fewer instructions
                    TileFlux<T, N> F{ub, hi, hasr[slot][q] ? ssl[slot][q] : nullptr, rbuf};
                    const int c = cidx(G, i, j, k);
                    const T resh2 = (F.div(i, j, k) - rt[q * V + c] * hh) * hh;
                    const T v = ub[c] + (T)(1.0 / 6.0) * resh2;
                    if (store) u[(int64_t)bid[slot][q] * V + c] = v;
                    if (keep) ub[c] = v;
                    const T a = resh2 < (T)0 ? -resh2 : resh2;
                    mt = a > mt ? a : mt;
                }
            };
            if constexpr (SW > 0) {
                // A thread's cell t has the same place in both colours: its
                // colour-1 cell and colour-2 cell are x neighbours.  Outside
                // reflux blocks their current values stay in registers
                // (own1, own2), so each colour loads only the other x
                // neighbour and the four y and z neighbours; the per-block
                // data is read once per tile.  This path only serves the mixed schedule's FP32
                // preconditioner, so it takes the cheaper form
                //   resh2 = (sum over faces of (u_nb - u_c)) (hi hh) - rhs hh^2
                // with explicit fused multiply-adds (hi hh = 1 up to
                // rounding); reflux blocks keep the reference's flux form.
                // rhs of this thread's two cells, read from the stage once per
                // launch when the launch does more than one sweep (with one
                // cell per colour: more would cost registers the occupancy
                // does not have)
                T own1[ITER], own2[ITER], th[ITER], ti[ITER], rr1[ITER], rr2[ITER];
                bool flux[ITER], live[ITER];
                int64_t gb[ITER];
#pragma unroll
                for (int x = 0; x < ITER; x++) {
                    const int t = ct + x * NCT, q = t / HALF;
                    live[x] = t < BPC * HALF && first + q < nblk;
                    if (live[x]) {
                        th[x] = shh[slot][q];
                        ti[x] = shi[slot][q];
                        flux[x] = hasr[slot][q] != 0;
                        gb[x] = (int64_t)bid[slot][q] * V;
                    }
                }
                bool have_rr2 = false;   // rr2 holds the colour-2 rhs (after the first colour-2 pass)
                auto fused_colour = [&](int pass, bool first_colour, bool keep, bool store) {
#pragma unroll
                    for (int x = 0; x < ITER; x++) {
                        if (!live[x]) continue;
                        int q, i1, j, k, d1;
                        cell_of(x, q, i1, j, k, d1);
                        const int dp = pass == 1 ? d1 : -d1;   // to this thread's other cell
                        const int i = pass == 1 ? i1 : i1 + d1;
                        const int c = cidx(G, i, j, k);
                        T *ub = ut + q * V;
                        T rr;
                        if constexpr (SW > 1 && ITER == 1) {
                            if (first_colour || (pass == 2 && !have_rr2)) {
                                rr = rt[q * V + c];
                                if (pass == 1) rr1[x] = rr;
                                else rr2[x] = rr;
                            } else {
                                rr = pass == 1 ? rr1[x] : rr2[x];
                            }
                        } else {
                            rr = rt[q * V + c];
                        }
                        T uc, resh2;
                        if (flux[x]) {
                            TileFlux<T, N> F{ub, ti[x], ssl[slot][q], rbuf};
                            uc = ub[c];
                            resh2 = (F.div(i, j, k) - rr * th[x]) * th[x];
                        } else {
                            T partner;
                            if (first_colour) {   // both cells still hold the values staged
                                uc = ub[c];
                                partner = ub[c + dp];
                                own2[x] = partner;
                            } else {
                                uc = pass == 1 ? own1[x] : own2[x];
                                partner = pass == 1 ? own2[x] : own1[x];
                            }
                            const T other = ub[c - dp];
                            const T ym = ub[c - G], yp = ub[c + G], zm = ub[c - G * G], zp = ub[c + G * G];
                            const T sx = (partner - uc) + (other - uc);
                            const T sy = (yp - uc) + (ym - uc);
                            const T sz = (zp - uc) + (zm - uc);
                            resh2 = fma((sx + sy) + sz, ti[x] * th[x], -(rr * (th[x] * th[x])));
                        }
                        const T v = fma((T)(1.0 / 6.0), resh2, uc);
                        if (pass == 1) own1[x] = v;
                        else own2[x] = v;
                        if (store) u[gb[x] + c] = v;
                        if (keep) ub[c] = v;
                        mt = fmax(mt, fabs(resh2));
                    }
                };
                if (got) fused_colour(1, true, true, SW == 1);
                // the consumer threads' barriers: each colour reads the
                // previous one's values from the stage; the first also ORs
                // the failed waits, so every consumer warp decides alike
                if (consumers_sync_or(1, NCT, !got)) {
                    if (ct == 0) atomicExch(&cab, 1);
                    break;
                }
#pragma unroll 1
                for (int r = 0; r < SW; r++) {
                    const bool last = r == SW - 1;
                    if (r > 0) {
                        fused_colour(1, false, true, last);
                        asm volatile("bar.sync 1, %0;" ::"r"(NCT) : "memory");
                    }
                    fused_colour(2, false, !last, last);
                    have_rr2 = true;
                    if (!last) asm volatile("bar.sync 1, %0;" ::"r"(NCT) : "memory");
                }
                // the stage held ordinary stores; the next bulk copy into it
                // goes through the async proxy
                fence_async_shared();
            } else {
                colour(ipass, false, true);
            }
            __syncwarp();
            if (lane == 0) {
                if (warp == 1) consumed[s]++;
                mbar_arrive(&empty[s]);   // this warp is done with stage s
            }
        }
        m = (double)mt;
    }
    __syncthreads();
    if (tid == 0 && (pab || cab)) {   // loads still in flight: wait for them (bounded), then report
        for (int s = 0; s < S; s++)
            for (int ph = consumed[s]; ph < issued[s]; ph++) mbar_wait_bounded(&full[s], (uint32_t)(ph & 1), kWaitPolls);
        atomicExch(err, 1);
    }
    cta_max_atomic(m, out);
}

// residual res = rhs - div F / h on listed blocks (fmg_poisson_resid)
// blocks per CTA of k_resid_tiled: two 8^3 blocks (1024 cells) measured
// faster than one
// (the default; the autotuner may choose 1, 2 or 4 for 8^3 blocks)
template <int N>
__host__ __device__ constexpr int resid_bpc() { return N == 8 ? 2 : Tile<N>::BPC; }
template <class TU, class TR, class TO, int N, int BPCX = resid_bpc<N>()>
__global__ void __launch_bounds__(256) k_resid_tiled(TO *__restrict__ res, const TU *__restrict__ u,
                                                     const TR *__restrict__ rhs, const int32_t *__restrict__ blocks,
                                                     int nblk, const double *__restrict__ h0,
                                                     const int32_t *__restrict__ level, const int32_t *__restrict__ rslot,
                                                     const double *__restrict__ rbuf, int f) {
    pdl_enter();
    using Tl = Tile<N>;
    constexpr int G = Tl::G, V = Tl::V, BPC = BPCX;
    __shared__ TU sh[BPC * V];
    __shared__ int ssl[BPC][6];
    __shared__ int sbid[BPC];
    __shared__ TU shi[BPC];
    __shared__ int8_t hasr[BPC];   // a face of the block takes a reflux flux
    const int first = blockIdx.x * BPC;
    stage_blocks<TU, N, BPC>(sh, u, blocks, first, nblk);
    if (threadIdx.x < BPC && first + (int)threadIdx.x < nblk) {   // per-block data, once per block
        const int q = threadIdx.x, b = blocks[first + q];
        int any = 0;
        for (int fc = 0; fc < 6; fc++) {
            const int v = rslot ? rslot[6 * b + fc] : -1;
            ssl[q][fc] = v;
            any |= v >= 0;
        }
        sbid[q] = b;
        hasr[q] = (int8_t)any;
        shi[q] = (TU)(1.0 / hlev(h0, level[b], f));
    }
    __syncthreads();
    for (int t = threadIdx.x; t < BPC * Tl::CELLS; t += blockDim.x) {
        const int q = t / Tl::CELLS, r = t - q * Tl::CELLS;
        if (first + q >= nblk) continue;
        const int i = r % N, j = (r / N) % N, k = r / (N * N);
        const TU hi = shi[q];
        TileFlux<TU, N> F{sh + q * V, hi, hasr[q] ? ssl[q] : nullptr, rbuf};
        const int64_t c = (int64_t)sbid[q] * V + cidx(G, i, j, k);
        res[c] = (TO)((TU)rhs[c] - F.div(i, j, k) * hi);
    }
}

// ---------------------------------------------------------------------------
// prolongation of listed blocks: fine level (N) interior from the same block
// one fmg level coarser (N/2 + 2 cells with ghosts), tricubic staged as
// interp_tricubic stages bufx / bufxy (interpolation.F90:98-217), or trilinear
// ---------------------------------------------------------------------------
// blocks per CTA of k_interp_tiled: at least 512 fine cells per CTA, and
// four 8^3 blocks (the per-CTA weights, load and three barriers amortised
// over more cells measured faster)
template <int N>
__host__ __device__ constexpr int interp_bpc() { return N == 8 ? 4 : (N * N * N >= 512 ? 1 : 512 / (N * N * N)); }
template <class T, int N>
__global__ void __launch_bounds__(256) k_interp_tiled(T *__restrict__ uf, const T *__restrict__ uc,
                                                      const int32_t *__restrict__ blocks, int nblk, int cubic) {
    pdl_enter();
    constexpr int NC = N / 2, GC = NC + 2, GF = N + 2;
    constexpr int VC = GC * GC * GC, VF = GF * GF * GF;
    constexpr int W = GC;                  // coarse extent with ghosts = interp range [-1, NC]
    constexpr int IB = interp_bpc<N>(), BX = N * W * W, BXY = N * N * W, NF = N * N * N;
    __shared__ T sc[IB * VC];
    __shared__ T bx[IB * BX];              // per block [kc][jc][i]
    __shared__ T bxy[IB * BXY];            // per block [kc][j][i]
    __shared__ int sb[IB];
    // Lagrange nodes and weights of fine index p (the same for x, y and z):
    // cubic_weights evaluated once per CTA instead of once per staged value
    __shared__ int cwc[N][4];
    __shared__ double cww[N][4];
    __shared__ T cwt[N][4];   // the weights rounded to T once (each use rounds them the same way)
    const int q0 = blockIdx.x * IB;
    const int nq = nblk - q0 < IB ? nblk - q0 : IB;
    if ((int)threadIdx.x < nq) sb[threadIdx.x] = blocks[q0 + threadIdx.x];
    if (threadIdx.x < N) {
        cubic_weights((int)threadIdx.x, -1, NC, cwc[threadIdx.x], cww[threadIdx.x]);
        for (int e = 0; e < 4; e++) cwt[threadIdx.x][e] = (T)cww[threadIdx.x][e];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nq * VC; t += blockDim.x) {
        const int q = t / VC;
        sc[t] = uc[(int64_t)sb[q] * VC + (t - q * VC)];
    }
    __syncthreads();
    if (!(cubic && NC + 2 >= 4)) {
        for (int t = threadIdx.x; t < nq * NF; t += blockDim.x) {
            const int q = t / NF, r = t - q * NF;
            const int i = r % N, j = (r / N) % N, k = r / (N * N);
            uf[(int64_t)sb[q] * VF + cidx(GF, i, j, k)] = trilinear_cell(sc + q * VC, GC, i, j, k, 0, 0, 0);
        }
        return;
    }
    // x: bx(i, jc, kc) for kc, jc in [-1, NC]
    for (int t = threadIdx.x; t < nq * BX; t += blockDim.x) {
        const int q = t / BX, r = t - q * BX;
        const int i = r % N, jc = (r / N) % W - 1, kc = r / (N * W) - 1;
        const int *c = cwc[i];
        const T *w = cwt[i];
        const T *row = sc + q * VC + cidx(GC, 0, jc, kc);
        bx[t] = w[0] * row[c[0]] + w[1] * row[c[1]] + w[2] * row[c[2]] + w[3] * row[c[3]];
    }
    __syncthreads();
    // y: bxy(i, j, kc)
    for (int t = threadIdx.x; t < nq * BXY; t += blockDim.x) {
        const int q = t / BXY, r = t - q * BXY;
        const int i = r % N, j = (r / N) % N, kc = r / (N * N) - 1;
        const int *c = cwc[j];
        const T *w = cwt[j];
        const T *bq = bx + q * BX;
        auto X = [&](int jc) { return bq[((kc + 1) * W + (jc + 1)) * N + i]; };
        bxy[t] = w[0] * X(c[0]) + w[1] * X(c[1]) + w[2] * X(c[2]) + w[3] * X(c[3]);
    }
    __syncthreads();
    // z
    for (int t = threadIdx.x; t < nq * NF; t += blockDim.x) {
        const int q = t / NF, r = t - q * NF;
        const int i = r % N, j = (r / N) % N, k = r / (N * N);
        const int *c = cwc[k];
        const T *w = cwt[k];
        const T *bq = bxy + q * BXY;
        auto Y = [&](int kc) { return bq[((kc + 1) * N + j) * N + i]; };
        uf[(int64_t)sb[q] * VF + cidx(GF, i, j, k)] = w[0] * Y(c[0]) + w[1] * Y(c[1]) + w[2] * Y(c[2]) + w[3] * Y(c[3]);
    }
}

// ---------------------------------------------------------------------------
// child -> parent restriction of one level: one CTA per BPC children
// ---------------------------------------------------------------------------
template <class T, int N>
__global__ void __launch_bounds__(256) k_converge_tiled(T *__restrict__ u, const int32_t *__restrict__ parent,
                                                        const int8_t *__restrict__ oct, int first, int nchild,
                                                        int cubic) {
    pdl_enter();
    using Tl = Tile<N>;
    constexpr int G = Tl::G, V = Tl::V, H = N / 2 > 0 ? N / 2 : 1, PER = H * H * H;
    constexpr int BPC = Tl::BPC;
    const int c0 = blockIdx.x * BPC;
    for (int t = threadIdx.x; t < BPC * PER; t += blockDim.x) {
        const int q = t / PER, r = t - q * PER;
        if (c0 + q >= nchild) continue;
        const int b = first + c0 + q;
        const int ic = r % H, jc = (r / H) % H, kc = r / (H * H);
        const T *uf = u + (int64_t)b * V;
        const T v = cubic ? rstrct_cubic(uf, G, 2 * ic, 2 * jc, 2 * kc) : rstrct_linear(uf, G, 2 * ic, 2 * jc, 2 * kc);
        u[(int64_t)parent[b] * V + cidx(G, ic + oct[3 * b] * H, jc + oct[3 * b + 1] * H, kc + oct[3 * b + 2] * H)] = v;
    }
}

// ---------------------------------------------------------------------------
// ordered FP64 sums: warps 1..31 stage the terms of the next chunk into shared
// memory (double-buffered) while thread 0 adds the current chunk in list
// order -- the same sequence of roundings as a single-thread loop, with the
// loads off its critical path.  One CTA of 1024 threads.
// ---------------------------------------------------------------------------
constexpr int kSumChunk = 1024;

// leaf mean: sum_b psum_b dv_b / sum_b n^3 dv_b over the listed blocks
__global__ void __launch_bounds__(1024) k_mean_combine_w(const double *__restrict__ psum,
                                                         const int32_t *__restrict__ blocks, int nblk,
                                                         const int32_t *__restrict__ level,
                                                         const double *__restrict__ h0, int n, double *out) {
    pdl_enter();
    __shared__ double tm[2][kSumChunk], tv[2][kSumChunk];
    const int tid = threadIdx.x;
    const double ncell = (double)(n * n * n);
    const int nch = (nblk + kSumChunk - 1) / kSumChunk;
    auto stage = [&](int c) {
        for (int t = tid - 32; t < kSumChunk; t += (int)blockDim.x - 32) {
            const int b = c * kSumChunk + t;
            if (b >= nblk) break;
            const double hd = h0[level[blocks[b]]];
            const double dv = hd * hd * hd;
            tm[c & 1][t] = psum[b] * dv;
            tv[c & 1][t] = ncell * dv;
        }
    };
    double mass = 0.0, vol = 0.0;
    if (tid >= 32 && nch > 0) stage(0);
    __syncthreads();
    for (int c = 0; c < nch; c++) {
        if (tid >= 32) {
            if (c + 1 < nch) stage(c + 1);
        } else if (tid == 0) {
            const int cnt = nblk - c * kSumChunk < kSumChunk ? nblk - c * kSumChunk : kSumChunk;
            for (int q = 0; q < cnt; q++) {
                mass = mass + tm[c & 1][q];
                vol = vol + tv[c & 1][q];
            }
        }
        __syncthreads();
    }
    if (tid == 0) *out = mass / vol;
}

// base-level average: sum_b psum_b / (n^3 nblk)
__global__ void __launch_bounds__(1024) k_ave_combine_w(const double *__restrict__ psum, int nblk, int n,
                                                        double *out) {
    pdl_enter();
    __shared__ double ts[2][kSumChunk];
    const int tid = threadIdx.x;
    const int nch = (nblk + kSumChunk - 1) / kSumChunk;
    auto stage = [&](int c) {
        for (int t = tid - 32; t < kSumChunk; t += (int)blockDim.x - 32) {
            const int b = c * kSumChunk + t;
            if (b >= nblk) break;
            ts[c & 1][t] = psum[b];
        }
    };
    double ave = 0.0;
    if (tid >= 32 && nch > 0) stage(0);
    __syncthreads();
    for (int c = 0; c < nch; c++) {
        if (tid >= 32) {
            if (c + 1 < nch) stage(c + 1);
        } else if (tid == 0) {
            const int cnt = nblk - c * kSumChunk < kSumChunk ? nblk - c * kSumChunk : kSumChunk;
            for (int q = 0; q < cnt; q++) ave = ave + ts[c & 1][q];
        }
        __syncthreads();
    }
    if (tid == 0) *out = nblk == 0 ? 0.0 : ave / (double)(n * n * n * nblk);
}

}  // namespace sfm
