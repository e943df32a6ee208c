// sfm_device.cuh -- device-side layout, index helpers and the batched
// per-element kernels of the FMG solve.
//
// Layout in HBM.  For every fmg sub-block level f (n = NI >> f cells per
// edge, G = n + 2 with the one ghost layer of fmg_data.F90:121) a field is
// one contiguous array [nblocks][G][G][G] (i fastest), blocks sorted by AMR
// level exactly as GridLevel(amr,fmg)%Block(gid) (fmg_data.F90:35-43) lists
// them.  Cell (i,j,k), -1 <= i,j,k <= n, of block b is at
// b*G^3 + ((k+1)*G + (j+1))*G + (i+1).
//
// Each kernel here is a functor applied to a flat range of work items by
// k_apply (one thread per output value, grid-stride).  Every functor
// evaluates its expression in the reference's order (Fortran left to right);
// the library is built with --fmad=false so FP64 results are bit-identical
// to the same expressions evaluated on the host.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sfm {

#define SFM_HD __host__ __device__ __forceinline__

// offset inside one block or the base grid (G <= 130: G^3 < 2^31); callers
// add it to a 64-bit block base
SFM_HD int cidx(int G, int i, int j, int k) { return ((k + 1) * G + (j + 1)) * G + (i + 1); }
// IJKC(i,0) = floor(i/2) (config.h:249)
SFM_HD int fdiv2(int i) { return i >= 0 ? i / 2 : -((-i + 1) / 2); }
// Fortran MODULO(i,2)
SFM_HD int modulo2(int i) { int r = i % 2; return r < 0 ? r + 2 : r; }
// NEAR(nf,nc) (interpolation.F90:55)
SFM_HD int near_(int nf, int nc) { return nc + 2 * modulo2(nf) - 1; }
// cell with coordinate `dir` = x and transverse coordinates (a,b), a on the lower axis
SFM_HD void put3(int dir, int x, int a, int b, int &i, int &j, int &k) {
    if (dir == 0) { i = x; j = a; k = b; }
    else if (dir == 1) { i = a; j = x; k = b; }
    else { i = a; j = b; k = x; }
}
SFM_HD int tra(int dir) { return dir == 0 ? 1 : 0; }   // lower transverse axis
SFM_HD int trb(int dir) { return dir == 2 ? 1 : 2; }   // upper transverse axis

// Lagrange weights of the 4-point cubic at fine index p inside a coarse
// buffer [lb, ub] (fmg_ghostcell.F90:577-598, interpolation.F90:106-127)
SFM_HD void cubic_weights(int p, int lb, int ub, int c[4], double a[4]) {
    int cP = fdiv2(p), cN = near_(p, cP);
    int c1 = cP < cN ? cP : cN, c2 = cP < cN ? cN : cP;
    int c0 = 2 * c1 - c2, c3 = 2 * c2 - c1;
    int nshift = 0;
    if (c3 > ub) nshift = c3 - ub;
    if (c0 < lb) nshift = c0 - lb;
    c0 -= nshift; c1 -= nshift; c2 -= nshift; c3 -= nshift;
    double xc = cP + 0.25 * (double)(2 * modulo2(p) - 1);
    a[0] = (xc - c1) * (xc - c2) * (xc - c3) / (double)((c0 - c1) * (c0 - c2) * (c0 - c3));
    a[1] = (xc - c0) * (xc - c2) * (xc - c3) / (double)((c1 - c0) * (c1 - c2) * (c1 - c3));
    a[2] = (xc - c0) * (xc - c1) * (xc - c3) / (double)((c2 - c0) * (c2 - c1) * (c2 - c3));
    a[3] = (xc - c0) * (xc - c1) * (xc - c2) / (double)((c3 - c0) * (c3 - c1) * (c3 - c2));
    c[0] = c0; c[1] = c1; c[2] = c2; c[3] = c3;
}

// ---------------------------------------------------------------------------
// device-resident hierarchy tables
// ---------------------------------------------------------------------------
struct FaceItem {          // one ghost face of one block for one pass
    int32_t dst, src;      // receiving block, source block (same level or parent level)
    int8_t lr, type;       // side; 0 same level copy, 1 coarse-fine interpolation
    int8_t oa, ob;         // octant bits of the receiver on the two transverse axes
};
struct RefluxItem {        // fine face whose neighbour is one level up (fmg_reflux.F90:143-163)
    int32_t fine, slot;    // fine block; coarse face slot receiving the mean flux
    int8_t dir, lr, oa, ob;
};
struct BFace {             // a (block, face) pair, e.g. a physical-boundary face
    int32_t b; int8_t face; int8_t pad[3];
};

struct Hier {
    int nb, nlev, NI, FMax;
    const int32_t *level;      // [nb]
    const int32_t *parent;     // [nb]
    const int8_t *oct;         // [3*nb] octant of each block in its parent
    const int8_t *skip;        // [nb] fmg_skip_grid (fmg_data.F90:618-628)
    const int32_t *rslot;      // [6*nb] reflux slot of a coarse face, -1 if none
    const double *h0;          // [nlev] cell width at fmg level 0
    const double *x0;          // [3*nb] centre of cell (0,0,0)
};

SFM_HD double hlev(const double *h0, int L, int f) { return h0[L] * (double)(1 << f); }

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
// Programmatic dependent launch: first statement of every kernel the solver
// launches with cudaLaunchAttributeProgrammaticStreamSerialization.  Such a
// grid is set up while the previous one drains (its CTAs are scheduled as
// the previous grid's CTAs exit) and waits here until that grid has
// completed with all its memory operations visible: the launch gap is
// hidden.  (Releasing the next grid early, at the start of this one,
// measured slower on the large levels.)  A no-op for a launch without the
// attribute.
__device__ __forceinline__ void pdl_enter() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
template <class Op>
__global__ void k_apply(Op op, int64_t n) {
    pdl_enter();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        op(i);
}

// element-wise op over whole listed blocks (functors with blocks, V and
// cell(c)): CTAs step over groups of bpc blocks, threads over their cells --
// no 64-bit division per element
template <class Op>
__global__ void __launch_bounds__(256) k_blocks(Op op, int nblk, int bpc) {
    pdl_enter();
    const int V = (int)op.V;
    for (int b0 = blockIdx.x * bpc; b0 < nblk; b0 += gridDim.x * bpc)
        for (int e = threadIdx.x; e < bpc * V; e += blockDim.x) {
            const int q = e / V, c = e - q * V;
            if (b0 + q < nblk) op.cell((int64_t)op.blocks[b0 + q] * V + c);
        }
}

// k_blocks in units of W values (V a multiple of W, arrays 16-byte aligned):
// one vector access per array and unit instead of W scalar ones
template <class Op, int W>
__global__ void __launch_bounds__(256) k_blocks_vec(Op op, int nblk, int bpc) {
    pdl_enter();
    const int VU = (int)op.V / W;
    for (int b0 = blockIdx.x * bpc; b0 < nblk; b0 += gridDim.x * bpc)
        for (int e = threadIdx.x; e < bpc * VU; e += blockDim.x) {
            const int q = e / VU, c = e - q * VU;
            if (b0 + q < nblk) op.template cells<W>((int64_t)op.blocks[b0 + q] * op.V + (int64_t)c * W);
        }
}

// Serial reference order for race checks: one thread per listed block
// applies op to the block's items per_block*q .. per_block*(q+1)-1 in order
// (the cell order of a single-threaded sweep), max of the results folded
// into *out as k_apply_max does.
template <class Op>
__global__ void k_serial_blocks(Op op, int nblk, int per_block, unsigned long long *out) {
    pdl_enter();
    double m = 0.0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nblk; q += gridDim.x * blockDim.x)
        for (int r = 0; r < per_block; r++) {
            const double v = op((int64_t)q * per_block + r);
            m = v > m ? v : m;
        }
    for (int o = 16; o > 0; o >>= 1) {
        double t = __shfl_xor_sync(0xffffffffu, m, o);
        m = t > m ? t : m;
    }
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// max over items of op(i) >= 0, folded into *out by atomicMax on the IEEE
// bit pattern (order-preserving for non-negative doubles)
template <class Op>
__global__ void k_apply_max(Op op, int64_t n, unsigned long long *out) {
    pdl_enter();
    double m = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double v = op(i);
        m = v > m ? v : m;
    }
    for (int o = 16; o > 0; o >>= 1) {
        double t = __shfl_xor_sync(0xffffffffu, m, o);
        m = t > m ? t : m;
    }
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// ---------------------------------------------------------------------------
// ghost cells (fmg_ghostcell.F90)
// ---------------------------------------------------------------------------
// One pass of fmg_ghostcell_fix for AMR level L and direction dir: the
// same-level face copies (fmg_ghfix_samelev, :127-199) and the coarse-fine
// interpolations (fmg_ghfix_parentlev, :312-496 bilinear, :506-733 bicubic)
// of that level.  Both write only the dir-ghost planes of level-L blocks and
// read only cells off those planes, so one launch holds both.
template <class T>
struct OpGhostPass {
    T *u; const FaceItem *items; int n, G; int64_t V; int dir, cubic;
    int sel;   // -1 both kinds, 0 same-level copies only, 1 coarse-fine only
    __device__ void operator()(int64_t idx) const {
        const int GT = n + 2;
        int64_t it = idx / (GT * GT);
        int r = (int)(idx - it * GT * GT);
        int p = r % GT - 1, q = r / GT - 1;
        FaceItem fi = items[it];
        if (sel >= 0 && fi.type != sel) return;
        T *ud = u + (int64_t)fi.dst * V;
        int xg = fi.lr == 0 ? -1 : n;
        int i, j, k;
        put3(dir, xg, p, q, i, j, k);
        if (fi.type == 0) {
            int xs = fi.lr == 0 ? n - 1 : 0, is, js, ks;
            put3(dir, xs, p, q, is, js, ks);
            ud[cidx(G, i, j, k)] = u[(int64_t)fi.src * V + cidx(G, is, js, ks)];
            return;
        }
        const T *uc = u + (int64_t)fi.src * V;
        const int nb2 = n / 2, xc = fi.lr == 0 ? n - 1 : 0;
        const int oa = fi.oa * nb2, ob = fi.ob * nb2;
        auto B = [&](int pb, int qb) -> T {
            int ci, cj, ck;
            put3(dir, xc, pb + oa, qb + ob, ci, cj, ck);
            return uc[cidx(G, ci, cj, ck)];
        };
        T uH;
        if (cubic && nb2 + 2 >= 4) {
            int cp[4], cq[4];
            double wp[4], wq[4];
            cubic_weights(p, -1, nb2, cp, wp);
            cubic_weights(q, -1, nb2, cq, wq);
            T bx[4];
#pragma unroll
            for (int m = 0; m < 4; m++)
                bx[m] = (T)wp[0] * B(cp[0], cq[m]) + (T)wp[1] * B(cp[1], cq[m]) + (T)wp[2] * B(cp[2], cq[m])
                      + (T)wp[3] * B(cp[3], cq[m]);
            uH = (T)wq[0] * bx[0] + (T)wq[1] * bx[1] + (T)wq[2] * bx[2] + (T)wq[3] * bx[3];
        } else {
            int pc = fdiv2(p), qc = fdiv2(q);
            int p1 = near_(p, pc), q1 = near_(q, qc);
            uH = ((T)9 * B(pc, qc) + B(p1, q1) + (T)3 * B(pc, q1) + (T)3 * B(p1, qc)) / (T)16;
        }
        int inner = fi.lr == 0 ? 1 : -1, i0, j0, k0, iN, jN, kN;
        put3(dir, xg + inner, p, q, i0, j0, k0);
        put3(dir, xg + 2 * inner, p, q, iN, jN, kN);
        T u0 = ud[cidx(G, i0, j0, k0)], uN = ud[cidx(G, iN, jN, kN)];
        ud[cidx(G, i, j, k)] = ((T)10 * u0 + (T)8 * uH - (T)3 * uN) / (T)15;
    }
};

// ---------------------------------------------------------------------------
// restriction (restriction.F90) and child->parent convergence
// (fmg_converge.F90:85-188)
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T rstrct_linear(const T *uf, int G, int i0, int j0, int k0) {
    const T rdv = (T)(1.0 / 8.0);
    return (uf[cidx(G, i0, j0, k0)] + uf[cidx(G, i0 + 1, j0, k0)]
          + uf[cidx(G, i0, j0 + 1, k0)] + uf[cidx(G, i0, j0, k0 + 1)]
          + uf[cidx(G, i0 + 1, j0 + 1, k0)] + uf[cidx(G, i0 + 1, j0, k0 + 1)]
          + uf[cidx(G, i0, j0 + 1, k0 + 1)] + uf[cidx(G, i0 + 1, j0 + 1, k0 + 1)]) * rdv;
}
// 1D weights {-1, 9, 9, -1} / 16 of the cubic restriction (exact in binary)
__device__ __forceinline__ double rstrct_w(int i) { return (i == 0 || i == 3) ? -1.0 / 16.0 : 9.0 / 16.0; }
template <class T>
__device__ __forceinline__ T rstrct_cubic(const T *uf, int G, int i1, int j1, int k1) {
    T s = (T)0;
#pragma unroll
    for (int kk = 0; kk < 4; kk++)
#pragma unroll
        for (int jj = 0; jj < 4; jj++)
#pragma unroll
            for (int ii = 0; ii < 4; ii++) {
                T t = uf[cidx(G, i1 - 1 + ii, j1 - 1 + jj, k1 - 1 + kk)] *
                      (T)((rstrct_w(ii) * rstrct_w(jj)) * rstrct_w(kk));
                s = (ii | jj | kk) ? s + t : t;
            }
    return s;
}

// every child of level Lf writes its restriction into its parent's octant
template <class T>
struct OpConverge {
    T *u; const int32_t *parent; const int8_t *oct; int first; int n, G; int64_t V; int cubic;
    __device__ void operator()(int64_t idx) const {
        const int h = n / 2, per = h * h * h;
        int b = first + (int)(idx / per);
        int r = (int)(idx % per);
        int ic = r % h, jc = (r / h) % h, kc = r / (h * h);
        const T *uf = u + (int64_t)b * V;
        T v = cubic ? rstrct_cubic(uf, G, 2 * ic, 2 * jc, 2 * kc) : rstrct_linear(uf, G, 2 * ic, 2 * jc, 2 * kc);
        int p = parent[b];
        u[(int64_t)p * V + cidx(G, ic + oct[3 * b] * h, jc + oct[3 * b + 1] * h, kc + oct[3 * b + 2] * h)] = v;
    }
};

// fmg_rstrct within each listed block: level f (nc cells) from f-1 (linear)
template <class TC, class TF>
struct OpRstrct {
    TC *uc; const TF *uf; const int32_t *blocks; int nc, Gc, Gf; int64_t Vc, Vf;
    __device__ void operator()(int64_t idx) const {
        const int per = nc * nc * nc;
        int b = blocks[idx / per];
        int r = (int)(idx % per);
        int ic = r % nc, jc = (r / nc) % nc, kc = r / (nc * nc);
        uc[(int64_t)b * Vc + cidx(Gc, ic, jc, kc)] = (TC)rstrct_linear(uf + (int64_t)b * Vf, Gf, 2 * ic, 2 * jc, 2 * kc);
    }
};

// ---------------------------------------------------------------------------
// prolongation (interpolation.F90)
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T trilinear_cell(const T *uc, int G, int ifn, int jf, int kf, int oi, int oj, int ok) {
    int icb = fdiv2(ifn), jcb = fdiv2(jf), kcb = fdiv2(kf);
    int ic = icb + oi, jc = jcb + oj, kc = kcb + ok;
    int ic1 = near_(ifn, icb) + oi, jc1 = near_(jf, jcb) + oj, kc1 = near_(kf, kcb) + ok;
    return ((T)27 * uc[cidx(G, ic, jc, kc)]
            + (T)9 * (uc[cidx(G, ic1, jc, kc)] + uc[cidx(G, ic, jc1, kc)] + uc[cidx(G, ic, jc, kc1)])
            + (T)3 * (uc[cidx(G, ic, jc1, kc1)] + uc[cidx(G, ic1, jc, kc1)] + uc[cidx(G, ic1, jc1, kc)])
            + uc[cidx(G, ic1, jc1, kc1)]) / (T)64;
}
// interp_tricubic for one fine cell of an n^3 block from the coarse array
// (buffer bounds [lb,ub] = [-1, nc]); the caller guarantees nc + 2 >= 4
// (nodes c* and weights w* of cubic_weights along each axis given)
template <class T>
__device__ __forceinline__ T tricubic_cell_w(const T *uc, int Gc, const int *ci, const double *wi, const int *cj,
                                             const double *wj, const int *ck, const double *wk) {
    T bxy[4];
#pragma unroll
    for (int mk = 0; mk < 4; mk++) {
        T bx[4];
#pragma unroll
        for (int mj = 0; mj < 4; mj++) {
            const T *row = uc + cidx(Gc, 0, cj[mj], ck[mk]);
            bx[mj] = (T)wi[0] * row[ci[0]] + (T)wi[1] * row[ci[1]] + (T)wi[2] * row[ci[2]] + (T)wi[3] * row[ci[3]];
        }
        bxy[mk] = (T)wj[0] * bx[0] + (T)wj[1] * bx[1] + (T)wj[2] * bx[2] + (T)wj[3] * bx[3];
    }
    return (T)wk[0] * bxy[0] + (T)wk[1] * bxy[1] + (T)wk[2] * bxy[2] + (T)wk[3] * bxy[3];
}
template <class T>
__device__ __forceinline__ T tricubic_cell(const T *uc, int Gc, int i, int j, int k, int lb, int ub) {
    int ci[4], cj[4], ck[4];
    double wi[4], wj[4], wk[4];
    cubic_weights(i, lb, ub, ci, wi);
    cubic_weights(j, lb, ub, cj, wj);
    cubic_weights(k, lb, ub, ck, wk);
    return tricubic_cell_w(uc, Gc, ci, wi, cj, wj, ck, wk);
}

// fmg_interp_cubic / fmg_interp_linear over the listed blocks (fmg.F90:826-843,
// fmg_interpol_cubic.F90:84-115): fine interior of level f from level f+1
template <class T>
struct OpInterp {
    T *uf; const T *uc; const int32_t *blocks; int n, Gf, Gc; int64_t Vf, Vc; int cubic;
    __device__ void operator()(int64_t idx) const {
        const int per = n * n * n;
        int b = blocks[idx / per];
        int r = (int)(idx % per);
        int i = r % n, j = (r / n) % n, k = r / (n * n);
        const T *c = uc + (int64_t)b * Vc;
        const int nc = n / 2;
        T v = (cubic && nc + 2 >= 4) ? tricubic_cell(c, Gc, i, j, k, -1, nc) : trilinear_cell(c, Gc, i, j, k, 0, 0, 0);
        uf[(int64_t)b * Vf + cidx(Gf, i, j, k)] = v;
    }
};

// vmg_interp_p2c_lev (vmg_interpol.F90:82-164): every child of level Lf
// gets its interior from the parent's octant (+1 ghost) by trilinear
template <class T>
struct OpP2C {
    T *uf; const T *uc; const int32_t *parent; const int8_t *oct; int first; int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int per = n * n * n;
        int b = first + (int)(idx / per);
        int r = (int)(idx % per);
        int i = r % n, j = (r / n) % n, k = r / (n * n);
        const int h = n / 2;
        uf[(int64_t)b * V + cidx(G, i, j, k)] =
            trilinear_cell(uc + (int64_t)parent[b] * V, G, i, j, k, oct[3 * b] * h, oct[3 * b + 1] * h, oct[3 * b + 2] * h);
    }
};

// ---------------------------------------------------------------------------
// physical boundary (fmg_boundary.F90)
// ---------------------------------------------------------------------------
template <class T>
struct OpFill0Faces {      // zero the listed ghost planes (whole transverse range)
    T *u; const BFace *faces; int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        // boundary faces x (n+2)^2 elements: far below 2^32
        const uint32_t GT = (uint32_t)n + 2, ui = (uint32_t)idx;
        const uint32_t it = ui / (GT * GT);
        int r = (int)(ui - it * GT * GT);
        BFace bf = faces[it];
        int dir = bf.face >> 1, lr = bf.face & 1, i, j, k;
        put3(dir, lr == 0 ? -1 : n, r % GT - 1, r / GT - 1, i, j, k);
        u[(int64_t)bf.b * V + cidx(G, i, j, k)] = (T)0;
    }
};
template <class T>
struct OpExtrapFaces {     // u_ghost = -u_inner for the listed faces of one direction
    T *u; const BFace *faces; int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        // boundary faces x (n+2)^2 elements: far below 2^32
        const uint32_t GT = (uint32_t)n + 2, ui = (uint32_t)idx;
        const uint32_t it = ui / (GT * GT);
        int r = (int)(ui - it * GT * GT);
        BFace bf = faces[it];
        int dir = bf.face >> 1, lr = bf.face & 1, i, j, k, ii, jj, kk;
        put3(dir, lr == 0 ? -1 : n, r % GT - 1, r / GT - 1, i, j, k);
        put3(dir, lr == 0 ? 0 : n - 1, r % GT - 1, r / GT - 1, ii, jj, kk);
        T *ub = u + (int64_t)bf.b * V;
        ub[cidx(G, i, j, k)] = -ub[cidx(G, ii, jj, kk)];
    }
};

// ---------------------------------------------------------------------------
// Poisson operator (fmg_poisson.F90)
// ---------------------------------------------------------------------------
// face flux F_dir at position x (between cell x and x+1) of block b,
// F = (u(x+1) - u(x)) / h (fmg_poisson.F90:102-108), replaced on a coarse
// face covered by finer blocks by the mean of the fine fluxes
// (fmg_reflux.F90:215-257) when reflux tables are given.
template <class T>
struct Flux {
    const T *ub; int G, n; T hi;
    const int32_t *rslot; const double *rbuf; int b;   // rslot == nullptr: no reflux
    __device__ __forceinline__ T operator()(int dir, int i, int j, int k) const {
        if (rslot) {
            int x = dir == 0 ? i : (dir == 1 ? j : k);
            if (x == n - 1 || x == -1) {
                int s = rslot[6 * b + (x == -1 ? 0 : 1) + 2 * dir];
                if (s >= 0) {
                    int a = dir == 0 ? j : i, c = dir == 2 ? j : k;
                    return (T)rbuf[(int64_t)s * n * n + (int64_t)c * n + a];
                }
            }
        }
        int i1 = i + (dir == 0), j1 = j + (dir == 1), k1 = k + (dir == 2);
        return (ub[cidx(G, i1, j1, k1)] - ub[cidx(G, i, j, k)]) * hi;
    }
    // divergence in the reference's left-to-right order
    __device__ __forceinline__ T div(int i, int j, int k) const {
        T t = (*this)(0, i, j, k) - (*this)(0, i - 1, j, k);
        t = t + (*this)(1, i, j, k);
        t = t - (*this)(1, i, j - 1, k);
        t = t + (*this)(2, i, j, k);
        t = t - (*this)(2, i, j, k - 1);
        return t;
    }
};

// fmg_reflux_do: mean of the 4 fine face fluxes per coarse face cell, in FP64
template <class T>
struct OpReflux {
    const T *u; const RefluxItem *items; double *rbuf; const double *h0; const int32_t *level; int f, n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        // items x (n/2)^2 elements: far below 2^32 (6 faces per block, n <= 16)
        const uint32_t h = (uint32_t)n / 2, per = h * h, ui = (uint32_t)idx;
        RefluxItem it = items[ui / per];
        int r = (int)(ui % per);
        int pc = r % h, qc = r / h;
        const T *ub = u + (int64_t)it.fine * V;
        double hd = hlev(h0, level[it.fine], f);
        T hi = (T)(1.0 / hd);
        int xf = it.lr == 0 ? -1 : n - 1;
        auto ff = [&](int p, int q) -> double {
            int i, j, k, i1, j1, k1;
            put3(it.dir, xf, p, q, i, j, k);
            put3(it.dir, xf + 1, p, q, i1, j1, k1);
            return (double)((ub[cidx(G, i1, j1, k1)] - ub[cidx(G, i, j, k)]) * hi);
        };
        int pf = 2 * pc, qf = 2 * qc;
        double v = (ff(pf, qf) + ff(pf, qf + 1) + ff(pf + 1, qf) + ff(pf + 1, qf + 1)) * 0.25;
        rbuf[(int64_t)it.slot * n * n + (int64_t)(qc + it.ob * h) * n + (pc + it.oa * h)] = v;
    }
};

// one colour of red-black Gauss-Seidel on the listed blocks
// (fmg_poisson_relax :160-211, vmg_poisson_relax vmg_poisson.F90:114-141);
// returns |resh2| for the max reduction
template <class T, class TR>
struct OpRelax {
    T *u; const TR *rhs; const int32_t *blocks; const double *h0; const int32_t *level;
    const int32_t *rslot; const double *rbuf; int f, n, G; int64_t V; int ipass;
    __device__ double operator()(int64_t idx) const {
        const int hn = n / 2, per = hn * n * n;
        int b = blocks[idx / per];
        int r = (int)(idx % per);
        int i2 = r % hn, j = (r / hn) % n, k = r / (hn * n);
        int i = 2 * i2 + ((j + k + ipass) & 1);
        double hd = hlev(h0, level[b], f);
        T hh = (T)hd, hi = (T)(1.0 / hd);
        T *ub = u + (int64_t)b * V;
        Flux<T> F{ub, G, n, hi, rslot, rbuf, b};
        int64_t c = cidx(G, i, j, k);
        T resh2 = (F.div(i, j, k) - (T)rhs[(int64_t)b * V + c] * hh) * hh;
        ub[c] = ub[c] + (T)(1.0 / 6.0) * resh2;
        return fabs((double)resh2);
    }
};

// fmg_poisson_resid (:217-265): res = rhs - div F / h on the listed blocks
template <class TU, class TR, class TO>
struct OpResid {
    TO *res; const TU *u; const TR *rhs; const int32_t *blocks; const double *h0; const int32_t *level;
    const int32_t *rslot; const double *rbuf; int f, n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int per = n * n * n;
        int b = blocks[idx / per];
        int r = (int)(idx % per);
        int i = r % n, j = (r / n) % n, k = r / (n * n);
        double hd = hlev(h0, level[b], f);
        TU hi = (TU)(1.0 / hd);
        Flux<TU> F{u + (int64_t)b * V, G, n, hi, rslot, rbuf, b};
        int64_t c = (int64_t)b * V + cidx(G, i, j, k);
        res[c] = (TO)((TU)rhs[c] - F.div(i, j, k) * hi);
    }
};

// |h^2 v| over the listed blocks' interiors (fmg_get_h2absmax, fmg.F90:1017-1039)
template <class T>
struct OpH2Abs {
    const T *a; const int32_t *blocks; const double *h0; const int32_t *level; int f, n, G; int64_t V;
    __device__ double operator()(int64_t idx) const {
        const int per = n * n * n;
        int b = blocks[idx / per];
        int r = (int)(idx % per);
        double hd = hlev(h0, level[b], f);
        return fabs((double)a[(int64_t)b * V + cidx(G, r % n, (r / n) % n, r / (n * n))]) * (hd * hd);
    }
};

// ---------------------------------------------------------------------------
// block-wise BLAS-1 over listed blocks, whole (G^3) arrays (fmg.F90:847-946,
// vmg.F90:509-563,682-706)
// ---------------------------------------------------------------------------
// W consecutive values as one 8- or 16-byte access (p aligned to W values)
template <class T, int W>
struct VecOf;
template <class T>
struct VecOf<T, 1> { using type = T; };
template <>
struct VecOf<float, 2> { using type = float2; };
template <>
struct VecOf<float, 4> { using type = float4; };
template <>
struct VecOf<double, 2> { using type = double2; };
template <class T, int W>
__device__ __forceinline__ void vec_load(const T *p, T (&v)[W]) {
    const typename VecOf<T, W>::type x = *reinterpret_cast<const typename VecOf<T, W>::type *>(p);
    const T *e = reinterpret_cast<const T *>(&x);
#pragma unroll
    for (int i = 0; i < W; i++) v[i] = e[i];
}
template <class T, int W>
__device__ __forceinline__ void vec_store(T *p, const T (&v)[W]) {
    typename VecOf<T, W>::type x;
    T *e = reinterpret_cast<T *>(&x);
#pragma unroll
    for (int i = 0; i < W; i++) e[i] = v[i];
    *reinterpret_cast<typename VecOf<T, W>::type *>(p) = x;
}
__host__ __device__ constexpr int vec_width(int bytes) { return 16 / bytes; }
inline bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }
// Each op also offers cells<W>(c): values c .. c+W-1 (one vector access per
// array, the same per-value expression), VW its widest W (16 bytes of its
// largest element type), aligned() whether its arrays allow vectors.
template <class TO, class TI>
struct OpCopy {
    TO *o; const TI *a; const int32_t *blocks; int64_t V;
    static constexpr int VW = vec_width(sizeof(TO) > sizeof(TI) ? sizeof(TO) : sizeof(TI));
    __device__ void operator()(int64_t idx) const { cell((int64_t)blocks[idx / V] * V + idx % V); }
    __device__ void cell(int64_t c) const { o[c] = (TO)a[c]; }
    template <int W>
    __device__ void cells(int64_t c) const {
        TI x[W];
        TO y[W];
        vec_load<TI, W>(a + c, x);
#pragma unroll
        for (int i = 0; i < W; i++) y[i] = (TO)x[i];
        vec_store<TO, W>(o + c, y);
    }
    bool aligned() const { return aligned16(o) && aligned16(a); }
};
template <class TA, class TD>
struct OpAdd {
    TA *a; const TD *d; const int32_t *blocks; int64_t V;
    static constexpr int VW = vec_width(sizeof(TA) > sizeof(TD) ? sizeof(TA) : sizeof(TD));
    __device__ void operator()(int64_t idx) const { cell((int64_t)blocks[idx / V] * V + idx % V); }
    __device__ void cell(int64_t c) const { a[c] = a[c] + (TA)d[c]; }
    template <int W>
    __device__ void cells(int64_t c) const {
        TA x[W];
        TD y[W];
        vec_load<TA, W>(a + c, x);
        vec_load<TD, W>(d + c, y);
#pragma unroll
        for (int i = 0; i < W; i++) x[i] = x[i] + (TA)y[i];
        vec_store<TA, W>(a + c, x);
    }
    bool aligned() const { return aligned16(a) && aligned16(d); }
};
template <class T>
struct OpSub {
    T *o; const T *a; const T *b_; const int32_t *blocks; int64_t V;
    static constexpr int VW = vec_width(sizeof(T));
    __device__ void operator()(int64_t idx) const { cell((int64_t)blocks[idx / V] * V + idx % V); }
    __device__ void cell(int64_t c) const { o[c] = a[c] - b_[c]; }
    template <int W>
    __device__ void cells(int64_t c) const {
        T x[W], y[W];
        vec_load<T, W>(a + c, x);
        vec_load<T, W>(b_ + c, y);
#pragma unroll
        for (int i = 0; i < W; i++) x[i] = x[i] - y[i];
        vec_store<T, W>(o + c, x);
    }
    bool aligned() const { return aligned16(o) && aligned16(a) && aligned16(b_); }
};
template <class T>
struct OpZero {
    T *o; const int32_t *blocks; int64_t V;
    static constexpr int VW = vec_width(sizeof(T));
    __device__ void operator()(int64_t idx) const { cell((int64_t)blocks[idx / V] * V + idx % V); }
    __device__ void cell(int64_t c) const { o[c] = (T)0; }
    template <int W>
    __device__ void cells(int64_t c) const {
        T x[W];
#pragma unroll
        for (int i = 0; i < W; i++) x[i] = (T)0;
        vec_store<T, W>(o + c, x);
    }
    bool aligned() const { return aligned16(o); }
};

}  // namespace sfm
