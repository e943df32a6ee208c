// sfm_solver.cu -- host driver of the B200 FMG Poisson solve and the C ABI
// of include/sfmg.h.
//
// The driver issues, in the reference's order, one batched kernel per
// operation of fmg_cycle / fmg_lin / vmg_fas (fmg.F90:134-377, vmg.F90:116-243):
// every block of a level (or of all levels) is updated by one launch driven
// from device-resident block, face and reflux tables; the base-grid solve
// (mg.F90:42-218) is one persistent CTA or a thread-block cluster.  All
// fields of all levels stay in HBM for the whole solve and across calls.
//
// Precision: Solver<double> is the plain FP64 path (bit-identical
// expressions to the reference's); Solver<float> runs fmg_lin and vmg_fas in
// FP32 inside the FP64 defect-correction loop, with the outer residual, the
// accumulation into phi, the reflux flux sums and the base-grid solve in FP64;
// its inner solve may follow a cheaper schedule than the reference's (the
// tuner's fused multi-sweep smoothing, fewer V-cycles), since it only
// preconditions the FP64 correction.
//
// Physical boundaries: periodic, isolated sphere, z-mirror sphere, MHD
// Bonnor-Ebert sphere and the z-periodic cylinders (fmg_boundary_phys_*.F90),
// each with its hooks at the reference's call sites.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <omp.h>
#if defined(__x86_64__)
#include <emmintrin.h>
#endif

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sfmg.h"
#include "sfm_device.cuh"
#include "sfm_kernels_misc.cuh"
#include "sfm_mg.cuh"
#include "sfm_fast.cuh"
#include "sfm_noalloc.cuh"
#include "sfm_adjoint.cuh"
#include "sfm_tune.h"

namespace sfm {

constexpr int Undef = -1;

// Runs BODY with a compile-time block edge N for the tiled kernels
// (N = 2, 4, 8, 16); other sizes take the per-element functors.
#define SFM_WITH_N(n, BODY, FALLBACK)                      \
    switch (n) {                                           \
        case 2: { constexpr int N = 2; BODY; } break;      \
        case 4: { constexpr int N = 4; BODY; } break;      \
        case 8: { constexpr int N = 8; BODY; } break;      \
        case 16: { constexpr int N = 16; BODY; } break;    \
        default: { FALLBACK; } break;                      \
    }

// ---------------------------------------------------------------------------
// host copy of the hierarchy, links and invariants
// (fmg_make_linklist fmg_data_if.F90:298-411, fmg_check_linklist :415-568)
// ---------------------------------------------------------------------------
struct HostHier {
    int nb = 0, nlev = 0, NI = 0, FMax = 0, ngb[3] = {0, 0, 0};
    std::vector<int> lstart, level, parent, child, nbr, nbrGid, baseIdx, ijk;
    std::vector<int8_t> oct, touch, sameLev, parLev, skip;
    std::vector<double> h0, x0;

    int build(const sfm_hier_desc *hd) {
        nb = hd->nblocks; nlev = hd->nlev; NI = hd->ni;
        if (nb <= 0 || nlev <= 0 || nlev > 30) return SFM_EINVAL;
        if (NI < 4 || (NI & (NI - 1)) || hd->nj != NI || hd->nk != NI || NI > 64) return SFM_EINVAL;
        if (!hd->level || !hd->ijk || !hd->parent || !hd->child || !hd->nbr || !hd->touch || !hd->cellwidth || !hd->x0)
            return SFM_EINVAL;
        for (int d = 0; d < 3; d++) { ngb[d] = hd->ngb[d]; if (ngb[d] <= 0) return SFM_EINVAL; }
        // The reference runs its serial base-grid multigrid whenever NGI/NGJ/
        // NGK_BASE are powers of two (vmg.F90:85-91), on boxes of any shape
        // (mg_data.F90:57-75, levels following min(boxsize)).  The base-grid
        // CTA here handles cubic boxes only, so a power-of-two box that is not
        // cubic is refused rather than solved by another method.
        {
            auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
            if (pow2(ngb[0]) && pow2(ngb[1]) && pow2(ngb[2]) && (ngb[0] != ngb[1] || ngb[1] != ngb[2]))
                return SFM_EHIER;
        }
        FMax = 0; while ((2 << FMax) < NI) FMax++;
        level.assign(hd->level, hd->level + nb);
        parent.assign(hd->parent, hd->parent + nb);
        child.assign(hd->child, hd->child + 8 * (size_t)nb);
        nbr.assign(hd->nbr, hd->nbr + 6 * (size_t)nb);
        ijk.assign(hd->ijk, hd->ijk + 3 * (size_t)nb);
        touch.resize(6 * (size_t)nb);
        for (size_t i = 0; i < touch.size(); i++) touch[i] = hd->touch[i] ? 1 : 0;
        h0.assign(hd->cellwidth, hd->cellwidth + nlev);
        x0.assign(hd->x0, hd->x0 + 3 * (size_t)nb);
        for (double v : h0) if (!(v > 0) || !std::isfinite(v)) return SFM_EINVAL;
        for (double v : x0) if (!std::isfinite(v)) return SFM_EINVAL;
        lstart.assign(nlev + 1, 0);
        for (int b = 0; b < nb; b++) {
            if (level[b] < 0 || level[b] >= nlev) return SFM_EHIER;
            if (b > 0 && level[b] < level[b - 1]) return SFM_EHIER;
            lstart[level[b] + 1]++;
        }
        for (int L = 0; L < nlev; L++) {
            lstart[L + 1] += lstart[L];
            if (lstart[L + 1] == lstart[L]) return SFM_EHIER;   // every level populated
        }
        for (int v : parent) if (v < -1 || v >= nb) return SFM_EHIER;
        for (int v : child) if (v < -1 || v >= nb) return SFM_EHIER;
        for (int v : nbr) if (v < -1 || v >= nb) return SFM_EHIER;
        // same-level and parent-level links
        nbrGid.assign(6 * (size_t)nb, Undef);
        sameLev.assign(6 * (size_t)nb, 0);
        parLev.assign(6 * (size_t)nb, 0);
        for (int b = 0; b < nb; b++)
            for (int f = 0; f < 6; f++)
                if (nbr[6 * b + f] != Undef) { nbrGid[6 * b + f] = nbr[6 * b + f]; sameLev[6 * b + f] = 1; }
        for (int L = 1; L < nlev; L++)
            for (int b = lstart[L]; b < lstart[L + 1]; b++) {
                int p = parent[b];
                if (p < 0) return SFM_EHIER;
                for (int f = 0; f < 6; f++) {
                    if (sameLev[6 * b + f]) continue;
                    int np = nbrGid[6 * p + f];
                    if (np == Undef) continue;
                    nbrGid[6 * b + f] = np;
                    parLev[6 * b + f] = 1;
                }
            }
        oct.assign(3 * (size_t)nb, 0);
        for (int b = 0; b < nb; b++) {
            if (level[b] == 0) { if (parent[b] != Undef) return SFM_EHIER; continue; }
            int p = parent[b], found = 0;
            for (int c = 0; c < 8; c++)
                if (child[8 * p + c] == b) {
                    oct[3 * b] = c & 1; oct[3 * b + 1] = (c >> 1) & 1; oct[3 * b + 2] = (c >> 2) & 1;
                    found++;
                }
            if (found != 1) return SFM_EHIER;
        }
        // invariants
        for (int b = 0; b < nb; b++) {
            int L = level[b];
            if (L > 0 && level[parent[b]] != L - 1) return SFM_EHIER;
            if (child[8 * b] != Undef) {
                if (L == nlev - 1) return SFM_EHIER;
                for (int c = 0; c < 8; c++) {
                    int cb = child[8 * b + c];
                    if (cb < 0 || parent[cb] != b || level[cb] != L + 1) return SFM_EHIER;
                }
            } else {
                for (int c = 1; c < 8; c++) if (child[8 * b + c] != Undef) return SFM_EHIER;
            }
            for (int f = 0; f < 6; f++) {
                int nbb = nbrGid[6 * b + f];
                if (sameLev[6 * b + f]) {
                    int fs = (f ^ 1);
                    if (level[nbb] != L || nbr[6 * nbb + fs] != b) return SFM_EHIER;
                    if (touch[6 * b + f]) return SFM_EHIER;
                }
                if (parLev[6 * b + f] && level[nbb] != L - 1) return SFM_EHIER;
                if ((int)sameLev[6 * b + f] + (int)parLev[6 * b + f] + (int)touch[6 * b + f] != 1) return SFM_EHIER;
            }
        }
        skip.assign(nb, 0);
        for (int b = 0; b < nb; b++) skip[b] = (level[b] != nlev - 1 && child[8 * b] != Undef) ? 1 : 0;
        baseIdx.assign((size_t)ngb[0] * ngb[1] * ngb[2], -1);
        if (lstart[1] != ngb[0] * ngb[1] * ngb[2]) return SFM_EHIER;
        for (int b = lstart[0]; b < lstart[1]; b++) {
            int i = hd->ijk[3 * b], j = hd->ijk[3 * b + 1], k = hd->ijk[3 * b + 2];
            if (i < 0 || j < 0 || k < 0 || i >= ngb[0] || j >= ngb[1] || k >= ngb[2]) return SFM_EHIER;
            int &slot = baseIdx[((size_t)k * ngb[1] + j) * ngb[0] + i];
            if (slot != -1) return SFM_EHIER;
            slot = b;
        }
        return SFM_OK;
    }
};

// ---------------------------------------------------------------------------
// device memory bookkeeping
// ---------------------------------------------------------------------------
// Guard bands (a debug mode, sfm_debug_set_guard_bytes): every device
// array of a context created while the setting is non-zero sits between two
// bands of that many bytes filled with kGuardByte; a kernel that writes
// past either end of an array changes a band (sfm_debug_check_guards counts
// the changed bytes), and one that reads past it reads NaN (0xFF bytes are
// a NaN in both float widths), which shows in the results.
constexpr unsigned char kGuardByte = 0xFF;
static std::atomic<uint64_t> g_guard_bytes{0};

struct DevMem {
    std::vector<void *> ptrs;
    int64_t bytes = 0;
    cudaError_t err = cudaSuccess;
    uint64_t guard = g_guard_bytes.load();
    struct Band { unsigned char *lo, *hi; size_t hiLen; };   // the bands below and above one array
    std::vector<Band> bands;
    template <class T>
    T *alloc(size_t count) {
        if (count == 0) count = 1;
        void *p = nullptr;
        const size_t payload = count * sizeof(T);
        if (guard > 0) {   // [band][payload rounded up to 256 B][band]
            const size_t body = (payload + 255) / 256 * 256;
            cudaError_t e = cudaMalloc(&p, body + 2 * guard);
            if (e != cudaSuccess) { err = e; return nullptr; }
            ptrs.push_back(p);
            unsigned char *base = static_cast<unsigned char *>(p);
            e = cudaMemset(base, kGuardByte, guard);
            if (e == cudaSuccess) e = cudaMemset(base + guard + payload, kGuardByte, body - payload + guard);
            if (e != cudaSuccess) { err = e; return nullptr; }
            bands.push_back({base, base + guard + payload, body - payload + guard});
            bytes += (int64_t)payload;
            return reinterpret_cast<T *>(base + guard);
        }
        cudaError_t e = cudaMalloc(&p, payload);
        if (e != cudaSuccess) { err = e; return nullptr; }
        ptrs.push_back(p);
        bytes += (int64_t)payload;
        return (T *)p;
    }
    // bytes of all bands that no longer hold kGuardByte (-1: a copy failed)
    int64_t guard_violations() const {
        int64_t bad = 0;
        std::vector<unsigned char> h;
        for (const Band &b : bands)
            for (int side = 0; side < 2; side++) {
                const size_t len = side ? b.hiLen : guard;
                h.resize(len);
                if (cudaMemcpy(h.data(), side ? b.hi : b.lo, len, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
                for (unsigned char v : h) bad += v != kGuardByte;
            }
        return bad;
    }
    template <class T>
    T *upload(const std::vector<T> &v) {
        T *p = alloc<T>(v.size());
        if (p && !v.empty()) {
            cudaError_t e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) err = e;
        }
        return p;
    }
    void release() {
        for (void *p : ptrs) cudaFree(p);
        ptrs.clear();
    }
};

struct Field {     // one element type, one fmg level, all blocks
    void *p = nullptr; int n = 0, G = 0; int64_t V = 0;
};

class SolverBase {
public:
    virtual ~SolverBase() {}
    virtual int solve(const double *rho, double *psi, double *g, sfm_stats *st, cudaStream_t s, int stop_stage,
                      double *dump) = 0;
    virtual int adjoint(const double *dJdphi, double *dJdrho, sfm_stats *st, cudaStream_t s) = 0;
    virtual int64_t device_bytes() const = 0;
    virtual int64_t guard_violations() const = 0;
    virtual int fmg_levels() const = 0;
    virtual void set_wait_polls(uint32_t polls) = 0;
    virtual void set_ghost_merge(bool on) = 0;
    virtual void set_serial_relax(bool on) = 0;
    virtual int autotune(int reps, const double *d_rho) = 0;
    virtual std::string tune_text() const = 0;
    virtual bool tune_load(const char *text) = 0;
    std::string last_error;
    // g written as [nblocks][3][ni^3] (block interiors only, no io ghost
    // layers) instead of the caller's layout: the host-array entry point
    // stages g this way
    bool gCompact = false;
    // io ghost width of rho and psi for this call (0: params.ngh_io); the
    // host-array entry point stages only the (-1:ni)^3 region the solve
    // reads and writes, a width of 1
    int ioGw = 0;
};

template <class T>
class Solver : public SolverBase {
public:
    HostHier H;
    sfm_params P;
    DevMem mem;
    cudaStream_t own_ = nullptr;   // the context's stream
    cudaStream_t st_ = nullptr;    // stream of the current call (caller's or own_)
    int64_t launches = 0;
    int maxBlocks = 148 * 16;
    int persistGrid = 148 * 8;   // CTAs of a persistent tiled sweep (set from the SM count in init)

    // device tables
    int32_t *d_level = nullptr, *d_parent = nullptr, *d_rslot = nullptr, *d_all = nullptr, *d_leaves = nullptr;
    int32_t *d_withChild = nullptr, *d_baseIdx = nullptr;
    int8_t *d_oct = nullptr, *d_skip = nullptr;
    double *d_h0 = nullptr, *d_x0 = nullptr;
    FaceItem *d_faces = nullptr;
    GFace *d_gface = nullptr;              // [6 nb] face types and sources for the level fills
    int32_t *d_kind26[3] = {nullptr, nullptr, nullptr};   // [sel + 1][26 nb] segment kinds (k_ghost_level)
    GItem *d_gitems = nullptr;             // general items of the level fills
    std::vector<std::array<int64_t, 3>> gOff;   // [level][sel + 1]: first general item
    std::vector<std::array<int, 3>> gCnt;       // [level][sel + 1]: general items
    std::vector<std::array<bool, 3>> ghostMerge;   // [level][sel + 1]: one launch fills the level
    int ghostForce = -1;                   // test hook: 1 / 0 forces the one-launch fill on / off, -1 the table
    bool serialRelax = false;              // test hook: colour sweeps one thread per block, in cell order
    TuneTable tune;                        // launch-shape choices (sfm_tune.h); empty = defaults
    // schedule of the inner solve: the reference's in FP64, the table's (if
    // any) in the mixed path, where the inner solve only preconditions the
    // FP64 defect correction
    int sched(int knob, int reference) const {
        return sizeof(T) == 4 ? tune.get(knob, 4, H.NI, -1, -1, reference) : reference;
    }
    RefluxItem *d_reflux = nullptr;
    BFace *d_tfL = nullptr, *d_tfDL = nullptr, *d_crop = nullptr;
    std::vector<int64_t> faceOff, faceSplit, tfLOff, tfDLOff, cropOff, wcOff;
    int32_t *d_zmin = nullptr;             // z-mirror: blocks touching the z-min face, level by level
    std::vector<int64_t> zminOff;
    double *d_cyllog = nullptr;            // z-periodic cylinders: ln(sqrt(x^2 + y^2)) at every ghost
                                           // cell of the boundary faces (d_tfL order), from the host's libm
    bool zperiodic() const { return P.bc == SFM_BC_CYL_ZPERIODIC || P.bc == SFM_BC_MASK_ZPERIODIC; }
    int nLeaves = 0, nReflux = 0, nSlots = 0;
    std::vector<int> leafList;

    // fields: inner precision T at every fmg level, FP64 outer fields at level 0
    std::vector<T *> U, RES, RHS, RHO;
    T *RUF = nullptr;
    double *SRC0 = nullptr, *PSI0 = nullptr, *PHI0 = nullptr, *RES0d = nullptr;
    std::vector<double *> rbuf;
    std::vector<int> nf, Gf;
    std::vector<int64_t> Vf;
    // scalars
    unsigned long long *d_max = nullptr;   // [8]
    double *d_scal = nullptr;              // [8]
    int *d_bad = nullptr;
    int *d_err = nullptr;                  // set by a device wait that gave up
    uint32_t waitPolls = kWaitPolls;       // poll limit of the smoother's stage waits (tests lower it)
    int nSM = 148;
    int bulkGrid[5][4][4] = {};            // persistent CTAs of k_relax_bulk<T, N, NT, SW>, by log2(N), NT, SW
    double *d_mom = nullptr, *d_part = nullptr, *d_psum = nullptr;
    int *d_mgit = nullptr;
    // base grid
    MgData mg;
    int mgSmemFrom = 0;
    size_t mgSmemBytes = 0;
    bool mgSmemOk = true;   // the opt-in to large dynamic shared memory succeeded
    bool mgFits[5][3] = {}; // a cluster of 2 << a CTAs with wide threshold 16 << b can be resident
    bool mg_fits(int nct, int wide) const {
        int a = -1, b = -1;
        for (int q = 0; q < 5; q++) if ((2 << q) == nct) a = q;
        for (int q = 0; q < 3; q++) if ((16 << q) == wide) b = q;
        return a >= 0 && b >= 0 && mgFits[a][b];
    }
    // Shared-memory plan of the base-grid launch.  wide = 0: one CTA, the
    // coarse levels that fit 200 KB in shared memory (never level 0).  wide > 0:
    // a cluster whose levels of at least `wide` cells per edge stay in global
    // memory, the smaller ones in CTA 0's shared memory as far as they fit,
    // plus every CTA's copy of the first small level when it is in shared
    // memory (it is interpolated onto a large level).
    struct MgPlan { int from; size_t bytes; int mirror; };
    MgPlan mg_plan(int wide) const {
        MgPlan pl{mg.MMax + 1, 0, 0};
        if (!mgSmemOk) return pl;
        size_t used = 0;
        int from = mg_smem_from(mg.N, mg.MMax, (size_t)200 * 1024 / sizeof(double), &used);
        int firstSmall = 0;
        if (wide > 0) {
            while (firstSmall <= mg.MMax && (mg.N >> firstSmall) >= wide) firstSmall++;
            if (from < firstSmall) {   // large levels stay in global memory
                from = firstSmall;
                used = 0;
                for (int m = from; m <= mg.MMax; m++) {
                    const size_t G = (size_t)(mg.N >> m) + 2;
                    used += 3 * G * G * G;
                }
            }
            if (firstSmall <= mg.MMax && firstSmall >= from) {
                const size_t G = (size_t)(mg.N >> firstSmall) + 2;
                pl.mirror = (int)(G * G * G);
            }
        }
        pl.from = from;
        pl.bytes = (used + (size_t)pl.mirror) * sizeof(double);
        return pl;
    }
    // the base-grid launch: one CTA, or a cluster of nct CTAs whose levels
    // of at least `wide` cells per edge use every CTA (level 0 must be one)
    void mg_launch(int nct, int wide) {
        const int nmax = sched(kKnobBaseCorr, 10);
        if (nct <= 1 || mg.N < wide || !mg_fits(nct, wide)) {
            launch_pdl(k_mg_cycle, 1, 512, mgSmemBytes, mg, mgSmemFrom, d_mgit, nmax, 1 << 30, 0);
            ++launches;
            return;
        }
        const MgPlan pl = mg_plan(wide);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(nct);
        cfg.blockDim = dim3(512);
        cfg.dynamicSmemBytes = pl.bytes;
        cfg.stream = st_;
        cudaLaunchAttribute at[2];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = nct;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 2;
        cudaLaunchKernelEx(&cfg, k_mg_cycle, mg, pl.from, d_mgit, nmax, wide, pl.mirror);
        ++launches;
    }
    // whether a cluster of nct CTAs with this plan can be resident
    bool mg_cluster_fits(int nct, int wide) {
        const MgPlan pl = mg_plan(wide);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(nct);
        cfg.blockDim = dim3(512);
        cfg.dynamicSmemBytes = pl.bytes;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = nct;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, (const void *)k_mg_cycle, &cfg) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return n >= 1;
    }
    bool useSerialMg = false;
    int NBc = 0;
    std::vector<std::pair<void *, size_t>> zeroList;   // re-zeroed at every solve
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    int FmgLevel_fill0 = Undef;

    // One defect-correction iteration of fmg_cycle (fmg.F90:183-185): the
    // FP64 composite residual, fmg_lin, and phi += u.  The launch sequence is
    // the same every iteration, so it is captured once as a CUDA graph and
    // replayed; without stream capture it runs eagerly.
    cudaGraphExec_t iterExec = nullptr;
    int64_t iterLaunches = 0;
    bool graphsOff = false;
    void outer_iteration_body() {
        nvtxRangePushA("sfm outer iteration");
        profNext = 0;
        resid<double, double, T>(0, RHO[0], PSI0, SRC0, false);
        fmg_lin();
        add(0, PSI0, U[0]);
        profPairs = profNext;
        nvtxRangePop();
    }
    void outer_iteration() {
        if (graphsOff) { outer_iteration_body(); return; }
        if (!iterExec) {
            int64_t l0 = launches;
            int save = FmgLevel_fill0;
            if (cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                cudaGetLastError();
                graphsOff = true;
                outer_iteration_body();
                return;
            }
            outer_iteration_body();
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(st_, &g);
            if (e == cudaSuccess) e = cudaGraphInstantiate(&iterExec, g, 0);
            if (g) cudaGraphDestroy(g);
            iterLaunches = launches - l0;
            launches = l0;
            FmgLevel_fill0 = save;
            if (e != cudaSuccess) {   // capture refused: run eagerly from now on
                cudaGetLastError();
                iterExec = nullptr;
                graphsOff = true;
                outer_iteration_body();
                return;
            }
        }
        cudaGraphLaunch(iterExec, st_);
        launches += iterLaunches;
        FmgLevel_fill0 = Undef;   // every iteration ends with a fresh flux at level 0
    }

    ~Solver() override {
        if (iterExec) cudaGraphExecDestroy(iterExec);
        prof_release();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (own_) cudaStreamDestroy(own_);
        mem.release();
    }
    int64_t device_bytes() const override { return mem.bytes; }
    int64_t guard_violations() const override { return mem.guard_violations(); }
    // the iteration graph holds the kernel parameters it was captured with:
    // a new limit drops it, and the next outer iteration captures again
    void set_serial_relax(bool on) override {
        serialRelax = on;
        if (iterExec) {
            cudaGraphExecDestroy(iterExec);
            iterExec = nullptr;
        }
    }
    void set_ghost_merge(bool on) override {
        ghostForce = on ? 1 : 0;
        if (iterExec) {
            cudaGraphExecDestroy(iterExec);
            iterExec = nullptr;
        }
    }
    // -----------------------------------------------------------------
    // Autotuner: times every candidate of every knob in use on this
    // context's hierarchy (each candidate `reps` times after one warm-up
    // launch, CUDA events on the context's stream, minimum kept) and keeps
    // the fastest in the table.  All candidates give bit-identical fields,
    // so the choice never changes a result; the reference's sweep counts and
    // coarse-level cutoff (fmg.F90:280-288, mg.F90:50-52, vmg.F90:85-91) are
    // not knobs, since they change the iterates.
    template <class F>
    float time_min(F &&op, int reps) {
        op();   // warm-up
        float best = std::numeric_limits<float>::max();
        for (int r = 0; r < reps; r++) {
            cudaEventRecord(ev0, st_);
            op();
            cudaEventRecord(ev1, st_);
            cudaEventSynchronize(ev1);
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess && ms < best) best = ms;
        }
        return best;
    }
    template <class TT>
    void tune_ghost(TT *u, int f, int sel, int reps) {
        const int n = nf[f];
        if (!(n == 2 || n == 4 || n == 8 || n == 16)) return;
        for (int L = 0; L < H.nlev; L++) {
            if (!ghostMerge[L][sel + 1] || (sel == 1 && L == 0)) continue;
            float t[2];
            for (int m = 0; m < 2; m++) {
                tune.set(kKnobGhostFill, (int)sizeof(TT), n, L, sel, m);
                t[m] = time_min([&] { ghost_fill_level(L, f, u, false, sel); }, reps);
            }
            tune.set(kKnobGhostFill, (int)sizeof(TT), n, L, sel, t[1] < t[0] ? 1 : 0);
        }
    }
    // Schedule of the mixed path's inner solve (see sfm_tune.h): coordinate
    // descent from the reference schedule over complete solves of the
    // caller's density, keeping a change only when the solve still reaches
    // rel_tol (stagnation exit and true residual as configured) and is at
    // least 2% faster.  The FP64 path keeps the reference's schedule.
    int tune_schedule(const double *d_rho, int reps) {
        auto solve_ms = [&](float &ms) -> bool {
            if (iterExec) {   // the graph holds the old schedule
                cudaGraphExecDestroy(iterExec);
                iterExec = nullptr;
            }
            sfm_stats st;
            const int rc = solve(d_rho, nullptr, nullptr, &st, own_, 0, nullptr);
            if (rc != SFM_OK || !(st.true_rel_residual <= P.rel_tol) || !st.converged) return false;
            ms = (float)st.device_ms;
            return true;
        };
        auto candidate = [&]() -> float {
            float ms = 0.f, best = std::numeric_limits<float>::max();
            if (!solve_ms(ms)) return best;   // the first solve also captures the graph
            for (int r = 0; r < reps; r++)
                if (solve_ms(ms) && ms < best) best = ms;
            return best;
        };
        struct Knob { int knob; int ref; std::vector<int> vals; };
        const Knob ks[] = {{kKnobFusedSweep, 0, {0, 1, 2, 3}},
                           {kKnobLocalSweeps, 1, {1, 2, 3}},
                           {kKnobBaseCorr, 10, {10, 4, 2, 1}},
                           {kKnobFmgCycles, 2, {2, 1}},
                           {kKnobFmgSweeps, 2, {2, 1, 3}},
                           {kKnobVmgSweeps, 2, {2, 1}}};
        for (const Knob &k : ks) tune.set(k.knob, 4, H.NI, -1, -1, k.ref);
        float best = candidate();
        if (best == std::numeric_limits<float>::max()) return SFM_ENOTCONVERGED;   // not even the reference
        // one round of coordinate descent (a second round, revisiting every
        // knob with the others at their new values, changed nothing on the
        // benchmark hierarchies and doubled the tuning time)
        for (const Knob &k : ks) {
            const int cur = tune.get(k.knob, 4, H.NI, -1, -1, k.ref);
            int pick = cur;
            for (int v : k.vals) {
                if (v == cur) continue;
                tune.set(k.knob, 4, H.NI, -1, -1, v);
                const float t = candidate();
                if (t < 0.98f * best) {
                    best = t;
                    pick = v;
                }
            }
            tune.set(k.knob, 4, H.NI, -1, -1, pick);
        }
        if (iterExec) {
            cudaGraphExecDestroy(iterExec);
            iterExec = nullptr;
        }
        return SFM_OK;
    }
    int autotune(int reps, const double *d_rho) override {
        st_ = own_;
        const int saveForce = ghostForce;
        ghostForce = -1;
        for (auto &z : zeroList) cudaMemsetAsync(z.first, 0, z.second, st_);
        FmgLevel_fill0 = Undef;
        const int FMax = H.FMax;
        // ghost fills: inner fields at every fmg level (both kinds), the
        // same-level and coarse-fine fills of the AMR-level V-cycle, and the
        // FP64 outer fields at fmg level 0
        for (int f = 0; f <= FMax; f++) tune_ghost<T>(U[f], f, -1, reps);
        tune_ghost<T>(U[FMax], FMax, 0, reps);
        tune_ghost<T>(U[FMax], FMax, 1, reps);
        if (sizeof(T) != sizeof(double)) tune_ghost<double>(PSI0, 0, -1, reps);
        // smoother CTA size on the bulk-copy levels: the two colour launches
        // (key kind -1) and, in the mixed path, the fused sweep (kind 1)
        for (int f = 0; f <= FMax; f++) {
            const int n = nf[f];
            bool bulk = false;
            SFM_WITH_N(n, bulk = bulk_ok<N>(), bulk = false)
            if (!bulk || nLeaves <= 0) continue;
            for (int kind : {-1, 1}) {
                const bool fused = kind == 1;
                if (fused && sizeof(T) != 4) continue;
                float best = std::numeric_limits<float>::max();
                int pick = n >= 16 ? 512 : 256;
                for (int nt : kRelaxNT) {
                    tune.set(kKnobRelaxThreads, (int)sizeof(T), n, -1, kind, nt);
                    const float t = time_min([&] {
                        for (int ipass = 1; ipass <= (fused ? 1 : 2); ipass++)
                            relax_launch(U[f], RHS[f], d_leaves, nLeaves, d_rslot, rbuf[f], f, ipass, d_max,
                                         fused ? 1 : 0);
                    }, reps);
                    if (t < best) { best = t; pick = nt; }
                }
                tune.set(kKnobRelaxThreads, (int)sizeof(T), n, -1, kind, pick);
            }
        }
        // residual blocks per CTA on 8^3 blocks (inner and outer precision)
        for (int f = 0; f <= FMax; f++) {
            if (nf[f] != 8) continue;
            const int cand[3] = {1, 2, 4};
            float best = std::numeric_limits<float>::max();
            int pick = 2;
            for (int c = 0; c < 3; c++) {
                tune.set(kKnobResidBpc, (int)sizeof(T), 8, -1, -1, cand[c]);
                const float t = time_min([&] {
                    FmgLevel_fill0 = f;   // time the residual kernel alone, not its ghost fill
                    resid<T, T, T>(f, RES[f], U[f], RHS[f], false);
                }, reps);
                if (t < best) { best = t; pick = cand[c]; }
            }
            tune.set(kKnobResidBpc, (int)sizeof(T), 8, -1, -1, pick);
            if (sizeof(T) != sizeof(double) && f == 0) {
                best = std::numeric_limits<float>::max();
                pick = 2;
                for (int c = 0; c < 3; c++) {
                    tune.set(kKnobResidBpc, 8, 8, -1, -1, cand[c]);
                    const float t = time_min([&] {
                        FmgLevel_fill0 = 0;
                        resid<double, double, T>(0, RHO[0], PSI0, SRC0, false);
                    }, reps);
                    if (t < best) { best = t; pick = cand[c]; }
                }
                tune.set(kKnobResidBpc, 8, 8, -1, -1, pick);
            }
        }
        // base-grid launch: one CTA or a cluster (same cells, same expressions)
        if (useSerialMg) {
            struct Cand { int nct, wide; };
            std::vector<Cand> cands = {{1, 16}};
            for (int nct : {2, 4, 8, 16})
                for (int w : {16, 32, 64})
                    if (NBc >= w && mg_fits(nct, w)) cands.push_back({nct, w});
            float best = std::numeric_limits<float>::max();
            Cand pick = {1, 16};
            for (const Cand &c : cands) {
                mg_launch(c.nct, c.wide);   // a launch the driver refuses is skipped
                if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st_) != cudaSuccess) {
                    cudaGetLastError();
                    continue;
                }
                const float t = time_min([&] { mg_launch(c.nct, c.wide); }, reps);
                if (t < best) {
                    best = t;
                    pick = c;
                }
            }
            tune.set(kKnobBaseCtas, (int)sizeof(T), NBc, -1, -1, pick.nct);
            tune.set(kKnobBaseWide, (int)sizeof(T), NBc, -1, -1, pick.wide);
        }
        FmgLevel_fill0 = Undef;
        if (iterExec) {   // the graph holds the old launch shapes
            cudaGraphExecDestroy(iterExec);
            iterExec = nullptr;
        }
        int rc = check("autotune");
        if (rc == SFM_OK && d_rho && sizeof(T) == 4) {
            rc = tune_schedule(d_rho, std::min(reps, 2));
            if (rc == SFM_OK) rc = check("autotune schedule");
        }
        ghostForce = saveForce;
        return rc;
    }
    std::string tune_text() const override { return tune.text(); }
    bool tune_load(const char *text) override {
        if (!tune.parse(text)) return false;
        if (iterExec) {
            cudaGraphExecDestroy(iterExec);
            iterExec = nullptr;
        }
        return true;
    }
    void set_wait_polls(uint32_t polls) override {
        waitPolls = polls;
        if (iterExec) {
            cudaGraphExecDestroy(iterExec);
            iterExec = nullptr;
        }
    }
    int fmg_levels() const override { return H.FMax + 1; }

    // -----------------------------------------------------------------
    int init(const sfm_hier_desc *hd, const sfm_params *p) {
        int rc = H.build(hd);
        if (rc) return rc;
        P = *p;
        if (cudaStreamCreateWithFlags(&own_, cudaStreamNonBlocking) != cudaSuccess) return SFM_ECUDA;
        st_ = own_;
        {
            int dev = 0, sms = 148;
            cudaGetDevice(&dev);
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
            persistGrid = sms * 8;
            nSM = sms;
            maxBlocks = sms * 16;
        }
        cudaEventCreate(&ev0);
        cudaEventCreate(&ev1);
        const int nb = H.nb, nlev = H.nlev, FMax = H.FMax;
        // ---- tables
        std::vector<int32_t> all(nb);
        for (int b = 0; b < nb; b++) all[b] = b;
        for (int b = 0; b < nb; b++) if (!H.skip[b]) leafList.push_back(b);
        nLeaves = (int)leafList.size();
        std::vector<int32_t> withChild;
        wcOff.assign(nlev + 1, 0);
        for (int L = 0; L < nlev; L++) {
            wcOff[L] = (int64_t)withChild.size();
            for (int b = H.lstart[L]; b < H.lstart[L + 1]; b++) if (H.child[8 * b] != Undef) withChild.push_back(b);
        }
        wcOff[nlev] = (int64_t)withChild.size();
        // ghost pass faces per (level, dir)
        std::vector<FaceItem> faces;
        faceOff.assign(nlev * 3 + 1, 0);
        for (int L = 0; L < nlev; L++)
            for (int dir = 0; dir < 3; dir++) {
                faceOff[L * 3 + dir] = (int64_t)faces.size();
                for (int b = H.lstart[L]; b < H.lstart[L + 1]; b++)
                    for (int lr = 0; lr < 2; lr++) {
                        int f = lr + 2 * dir;
                        if (!H.sameLev[6 * b + f] && !(L > 0 && H.parLev[6 * b + f])) continue;
                        FaceItem it;
                        it.dst = b; it.src = H.nbrGid[6 * b + f]; it.lr = (int8_t)lr;
                        it.type = H.sameLev[6 * b + f] ? 0 : 1;
                        it.oa = H.oct[3 * b + tra(dir)]; it.ob = H.oct[3 * b + trb(dir)];
                        faces.push_back(it);
                    }
                // Items of one pass are independent (a pass writes only ghost
                // cells of its direction and reads none), so their order is
                // free.  A block's row-boundary sectors hold its ghosts and its
                // boundary planes on both sides, touched by the two faces it
                // shares with each neighbour: same-level pairs are ordered
                // along each line of blocks in the pass direction, so
                // consecutive pairs meet those sectors while they are in L2;
                // the fine faces under one coarse face follow each other.
                auto key = [&](const FaceItem &x) -> int64_t {
                    if (x.type != 0) return ((int64_t)1 << 62) | ((int64_t)x.src << 8);
                    const int lo = H.ijk[3 * x.dst + dir] <= H.ijk[3 * x.src + dir] ? x.dst : x.src;
                    const int64_t ta = H.ijk[3 * lo + tra(dir)], tb = H.ijk[3 * lo + trb(dir)];
                    return (ta << 42) | (tb << 21) | (int64_t)H.ijk[3 * lo + dir];
                };
                std::stable_sort(faces.begin() + faceOff[L * 3 + dir], faces.end(),
                                 [&](const FaceItem &a, const FaceItem &c) { return key(a) < key(c); });
            }
        faceOff[nlev * 3] = (int64_t)faces.size();
        // each list holds its same-level items first (key bit 62 marks
        // coarse-fine ones): faceSplit is where the coarse-fine ones start
        faceSplit.assign(nlev * 3, 0);
        for (int k = 0; k < nlev * 3; k++) {
            int64_t i = faceOff[k];
            while (i < faceOff[k + 1] && faces[i].type == 0) i++;
            faceSplit[k] = i;
        }
        // reflux: coarse faces covered by finer blocks get a slot
        std::vector<int32_t> rslot(6 * (size_t)nb, -1);
        std::vector<RefluxItem> refl;
        for (int L = 1; L < nlev; L++)
            for (int b = H.lstart[L]; b < H.lstart[L + 1]; b++)
                for (int dir = 0; dir < 3; dir++)
                    for (int lr = 0; lr < 2; lr++) {
                        int f = lr + 2 * dir;
                        if (!H.parLev[6 * b + f]) continue;
                        int cb = H.nbrGid[6 * b + f];
                        int cf = (1 - lr) + 2 * dir;   // the coarse block's face
                        if (rslot[6 * cb + cf] < 0) rslot[6 * cb + cf] = nSlots++;
                        RefluxItem it;
                        it.fine = b; it.slot = rslot[6 * cb + cf]; it.dir = (int8_t)dir; it.lr = (int8_t)lr;
                        it.oa = H.oct[3 * b + tra(dir)]; it.ob = H.oct[3 * b + trb(dir)];
                        refl.push_back(it);
                    }
        nReflux = (int)refl.size();
        // physical-boundary faces, by level then dir, and by dir then level
        std::vector<BFace> tfL, tfDL;
        tfLOff.assign(nlev + 1, 0);
        for (int L = 0; L < nlev; L++) {
            tfLOff[L] = (int64_t)tfL.size();
            for (int dir = 0; dir < 3; dir++)
                for (int b = H.lstart[L]; b < H.lstart[L + 1]; b++)
                    for (int lr = 0; lr < 2; lr++)
                        if (H.touch[6 * b + lr + 2 * dir]) { BFace x{}; x.b = b; x.face = (int8_t)(lr + 2 * dir); tfL.push_back(x); }
        }
        tfLOff[nlev] = (int64_t)tfL.size();
        tfDLOff.assign(3 * nlev + 1, 0);
        for (int dir = 0; dir < 3; dir++)
            for (int L = 0; L < nlev; L++) {
                tfDLOff[dir * nlev + L] = (int64_t)tfDL.size();
                for (int b = H.lstart[L]; b < H.lstart[L + 1]; b++)
                    for (int lr = 0; lr < 2; lr++)
                        if (H.touch[6 * b + lr + 2 * dir]) { BFace x{}; x.b = b; x.face = (int8_t)(lr + 2 * dir); tfDL.push_back(x); }
            }
        tfDLOff[3 * nlev] = (int64_t)tfDL.size();
        // tau crop faces per child level
        std::vector<BFace> crop;
        cropOff.assign(nlev + 1, 0);
        for (int L = 0; L < nlev; L++) {
            cropOff[L] = (int64_t)crop.size();
            if (L == 0) continue;
            for (int b = H.lstart[L]; b < H.lstart[L + 1]; b++)
                for (int f = 0; f < 6; f++)
                    if (H.parLev[6 * b + f]) { BFace x{}; x.b = b; x.face = (int8_t)f; crop.push_back(x); }
        }
        cropOff[nlev] = (int64_t)crop.size();

        // faces of every block for the level fills, and which fills of which
        // level one launch can do
        std::vector<GFace> gface(6 * (size_t)nb);
        for (int b = 0; b < nb; b++)
            for (int fc = 0; fc < 6; fc++) {
                GFace g{};
                g.src = H.nbrGid[6 * b + fc];
                g.type = H.sameLev[6 * b + fc] ? 0 : (H.level[b] > 0 && H.parLev[6 * b + fc] ? 1 : 2);
                if (g.type == 2) g.src = -1;
                gface[6 * b + fc] = g;
            }
        ghostMerge.assign(nlev, {false, false, false});
        for (int L = 0; L < nlev; L++)
            for (int sel = -1; sel <= 1; sel++) ghostMerge[L][sel + 1] = ghost_merge_ok(gface, L, sel);
        // segment kinds and general items of the exact level fills (see kind26)
        std::vector<GItem> gitems;
        std::array<std::vector<int32_t>, 3> kind26;
        gOff.assign(nlev, {});
        gCnt.assign(nlev, {});
        for (int sel = -1; sel <= 1; sel++) kind26[sel + 1].assign(26 * (size_t)nb, kSegSkip);
        for (int L = 0; L < nlev; L++)
            for (int sel = -1; sel <= 1; sel++) {
                gOff[L][sel + 1] = (int64_t)gitems.size();
                if (ghostMerge[L][sel + 1])
                    for (int b = H.lstart[L]; b < H.lstart[L + 1]; b++)
                        for (int seg = 0; seg < 26; seg++) {
                            int sg[3];
                            segment_sides(seg, sg[0], sg[1], sg[2]);
                            const int nz = (sg[0] != 0) + (sg[1] != 0) + (sg[2] != 0);
                            bool written = false;
                            for (int d = 0; d < 3; d++)
                                if (sg[d] && gface_filled(gface[6 * b + (sg[d] > 0) + 2 * d].type, sel)) written = true;
                            int32_t kind = kSegSkip;
                            if (written) {
                                int cur = b;   // the chain of the passes through same-level faces only
                                for (int d = 2; d >= 0 && cur >= 0; d--) {
                                    if (!sg[d]) continue;
                                    const GFace &g = gface[6 * cur + (sg[d] > 0) + 2 * d];
                                    cur = (g.type == 0 && gface_filled(0, sel)) ? g.src : -1;
                                }
                                if (cur >= 0) {
                                    kind = cur;
                                } else if (nz == 1) {   // a filled coarse-fine face
                                    kind = kSegCF;
                                } else {
                                    kind = kSegGeneral;
                                    GItem e{};
                                    e.dst = b;
                                    e.seg = (int8_t)seg;
                                    gitems.push_back(e);
                                }
                            }
                            kind26[sel + 1][26 * (size_t)b + seg] = kind;
                        }
                gCnt[L][sel + 1] = (int)((int64_t)gitems.size() - gOff[L][sel + 1]);
            }
        d_level = mem.upload(std::vector<int32_t>(H.level.begin(), H.level.end()));
        d_parent = mem.upload(std::vector<int32_t>(H.parent.begin(), H.parent.end()));
        d_oct = mem.upload(H.oct);
        d_skip = mem.upload(H.skip);
        d_rslot = mem.upload(rslot);
        d_h0 = mem.upload(H.h0);
        d_x0 = mem.upload(H.x0);
        d_all = mem.upload(all);
        d_leaves = mem.upload(std::vector<int32_t>(leafList.begin(), leafList.end()));
        d_withChild = mem.upload(withChild);
        d_faces = mem.upload(faces);
        d_gface = mem.upload(gface);
        d_gitems = mem.upload(gitems);
        for (int q = 0; q < 3; q++) d_kind26[q] = mem.upload(kind26[q]);
        d_reflux = mem.upload(refl);
        d_tfL = mem.upload(tfL);
        if (zperiodic()) {   // the cylinders' ghost values are a00 times these (x and y faces only)
            const int n = H.NI, GT = n + 2;
            std::vector<double> lg((size_t)tfL.size() * GT * GT, 0.0);
            for (size_t it = 0; it < tfL.size(); it++) {
                const int b = tfL[it].b, dir = tfL[it].face >> 1, lr = tfL[it].face & 1;
                if (dir == 2) continue;
                const double hb = H.h0[H.level[b]];
                for (int r = 0; r < GT * GT; r++) {
                    int i, j, k;
                    put3(dir, lr == 0 ? -1 : n, r % GT - 1, r / GT - 1, i, j, k);
                    const double x = H.x0[3 * b] + (double)i * hb, y = H.x0[3 * b + 1] + (double)j * hb;
                    lg[it * GT * GT + r] = std::log(std::sqrt(x * x + y * y));
                }
            }
            d_cyllog = mem.upload(lg);
        }
        {   // z-mirror plane (TouchBoundary(Left, MZ)), per AMR level
            std::vector<int32_t> zm;
            zminOff.assign(nlev + 1, 0);
            for (int L = 0; L < nlev; L++) {
                zminOff[L] = (int64_t)zm.size();
                if (P.bc == SFM_BC_ZMIRROR)
                    for (int b = H.lstart[L]; b < H.lstart[L + 1]; b++)
                        if (H.touch[6 * b + 4]) zm.push_back(b);
            }
            zminOff[nlev] = (int64_t)zm.size();
            d_zmin = mem.upload(zm);
        }
        d_tfDL = mem.upload(tfDL);
        d_crop = mem.upload(crop);
        d_baseIdx = mem.upload(std::vector<int32_t>(H.baseIdx.begin(), H.baseIdx.end()));
        // ---- fields
        nf.resize(FMax + 1); Gf.resize(FMax + 1); Vf.resize(FMax + 1);
        for (int f = 0; f <= FMax; f++) { nf[f] = H.NI >> f; Gf[f] = nf[f] + 2; Vf[f] = (int64_t)Gf[f] * Gf[f] * Gf[f]; }
        auto fieldT = [&](int f) { T *p = mem.alloc<T>((size_t)nb * Vf[f]); zeroList.push_back({p, (size_t)nb * Vf[f] * sizeof(T)}); return p; };
        auto fieldD = [&](int f) { double *p = mem.alloc<double>((size_t)nb * Vf[f]); zeroList.push_back({p, (size_t)nb * Vf[f] * sizeof(double)}); return p; };
        for (int f = 0; f <= FMax; f++) {
            U.push_back(fieldT(f)); RES.push_back(fieldT(f)); RHS.push_back(fieldT(f)); RHO.push_back(fieldT(f));
            rbuf.push_back(mem.alloc<double>((size_t)std::max(nSlots, 1) * nf[f] * nf[f]));
        }
        RUF = fieldT(FMax);
        SRC0 = fieldD(0); PSI0 = fieldD(0); PHI0 = fieldD(0); RES0d = fieldD(0);
        d_max = mem.alloc<unsigned long long>(8);
        d_scal = mem.alloc<double>(8);
        d_bad = mem.alloc<int>(1);
        d_err = mem.alloc<int>(1);
        zeroList.push_back({d_err, sizeof(int)});
        for (int f = 0; f <= FMax; f++) SFM_WITH_N(nf[f], bulk_grids<N>(), (void)0);
        d_mom = mem.alloc<double>(32);
        if (P.bc != SFM_BC_PERIODIC)   // per-cell moment terms of the base level, summed in order
            d_part = mem.alloc<double>((size_t)H.lstart[1] * H.NI * H.NI * H.NI * kMomentTerms);
        d_psum = mem.alloc<double>((size_t)nb);
        d_mgit = mem.alloc<int>(1);
        // ---- base grid (mg_data_init, mg_data.F90:45-90)
        auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
        int NBx = (H.ngb[0] * H.NI) >> FMax, NBy = (H.ngb[1] * H.NI) >> FMax, NBz = (H.ngb[2] * H.NI) >> FMax;
        // UseSerialMg (vmg.F90:85-91); non-cubic power-of-two boxes were refused in HostHier::build
        useSerialMg = pow2(H.ngb[0]) && pow2(H.ngb[1]) && pow2(H.ngb[2]) && NBx == NBy && NBy == NBz;
        std::memset(&mg, 0, sizeof(mg));
        if (useSerialMg) {
            NBc = NBx;
            int MMax = 0; while ((1 << MMax) < NBc) MMax++;
            if (MMax + 1 > MG_MAXLEV) return SFM_ESIZE;
            mg.N = NBc; mg.MMax = MMax;
            mg.hbase = hlev(H.h0.data(), 0, FMax);
            mg.periodic = P.bc == SFM_BC_PERIODIC ? 1 : 0;
            mg.zbc = P.bc == SFM_BC_ZMIRROR ? 1 : (zperiodic() ? 2 : 0);
            for (int f = 0; f < 6; f++) {
                mg.touch[f] = 0;
                for (int b = H.lstart[0]; b < H.lstart[1]; b++) mg.touch[f] |= H.touch[6 * b + f];
            }
            for (int m = 0; m <= MMax; m++) {
                size_t G = (size_t)(NBc >> m) + 2, V = G * G * G;
                mg.U[m] = mem.alloc<double>(V); mg.RES[m] = mem.alloc<double>(V);
                mg.RHS[m] = mem.alloc<double>(V); mg.RHO[m] = mem.alloc<double>(V);
                for (double *q : {mg.U[m], mg.RES[m], mg.RHS[m], mg.RHO[m]}) zeroList.push_back({q, V * sizeof(double)});
            }
            // shared-memory plans of the one-CTA launch and of the cluster
            // launches (one per wide threshold); opt in to the largest,
            // whatever the size: static and dynamic together may pass 48 KB
            size_t most = 0;
            for (int w : {0, 16, 32, 64}) most = std::max(most, mg_plan(w).bytes);
            bool optin = cudaFuncSetAttribute(k_mg_cycle, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most) ==
                         cudaSuccess;
            if (!optin) cudaGetLastError();
            mgSmemOk = optin;
            if (cudaFuncSetAttribute(k_mg_cycle, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
                cudaGetLastError();
            const MgPlan one = mg_plan(0);
            mgSmemFrom = one.from;
            mgSmemBytes = one.bytes;
            // which cluster shapes can be resident, asked once here (outside
            // any stream capture); a table may only pick among these
            for (int a = 0; a < 5; a++)
                for (int b = 0; b < 3; b++) mgFits[a][b] = mg_cluster_fits(2 << a, 16 << b);
            size_t G0 = (size_t)NBc + 2, V0 = G0 * G0 * G0;
            mg.SRC = mem.alloc<double>(V0); mg.PSI = mem.alloc<double>(V0);
            zeroList.push_back({mg.SRC, V0 * sizeof(double)});
            zeroList.push_back({mg.PSI, V0 * sizeof(double)});
        }
        if (mem.err != cudaSuccess) {
            last_error = cudaGetErrorString(mem.err);
            return mem.err == cudaErrorMemoryAllocation ? SFM_ENOMEM : SFM_ECUDA;
        }
        return SFM_OK;
    }

    // -----------------------------------------------------------------
    // launch helpers
    // Every kernel of the solve starts with pdl_enter(), so each launch
    // carries a programmatic dependency on the previous kernel of the
    // stream: it is scheduled while that one drains.  (Chained this way,
    // separate launches measured faster than one cooperative launch per
    // small-level relax with grid barriers between its phases: nested5 89
    // -> 67 ms.)
    template <class... KArgs, class... Args>
    void launch_pdl(void (*k)(KArgs...), unsigned grid, unsigned block, size_t smem, Args... args) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(block);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st_;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, k, args...);
    }
    template <class Op>
    void run(const Op &op, int64_t n) {
        if (n <= 0) return;
        int64_t blocks = (n + 255) / 256;
        if (blocks > maxBlocks) blocks = maxBlocks;
        launch_pdl(k_apply<Op>, (unsigned)blocks, 256, 0, op, n);
        ++launches;
    }
    template <class Op>
    void runMax(const Op &op, int64_t n, unsigned long long *out) {
        if (n <= 0) return;
        int64_t blocks = (n + 255) / 256;
        if (blocks > maxBlocks) blocks = maxBlocks;
        launch_pdl(k_apply_max<Op>, (unsigned)blocks, 256, 0, op, n, out);
        ++launches;
    }
    int cnt(int L) const { return H.lstart[L + 1] - H.lstart[L]; }

    // -----------------------------------------------------------------
    // Whether k_ghost_level fills level L (fill kind sel) exactly as the
    // three passes do.  The kernel evaluates each shell cell's final value
    // by the composition the passes apply (highest filled ghost dimension
    // first, then the cells that pass reads, dimension by dimension); where
    // that composition reads a ghost cell no earlier pass wrote, it reads
    // memory, which is exact only if no pass of this fill writes that cell
    // at all.  The same recursion is walked here on every block of the level
    // and for each of its 26 shell segments (a segment's cells share one
    // recursion: which coordinates are ghosts and on which side).
    bool ghost_merge_ok(const std::vector<GFace> &gf, int L, int sel) const {
        auto filled = [&](int b, int d, int side) { return gface_filled(gf[6 * b + (side > 0) + 2 * d].type, sel); };
        bool race = false;
        // state of segment s (per dimension -1 low ghost, 0 interior, 1 high ghost) of block b after passes 0..dl
        auto walk = [&](auto &&self, int b, std::array<int, 3> sg, int dl) -> void {
            for (int d = dl; d >= 0; d--) {
                if (sg[d] == 0 || !filled(b, d, sg[d])) continue;
                const GFace &g = gf[6 * b + (sg[d] > 0) + 2 * d];
                std::array<int, 3> s2 = sg;
                s2[d] = 0;
                self(self, g.type == 0 ? g.src : b, s2, d - 1);   // same level: the neighbour; coarse-fine: u0, uN
                return;
            }
            for (int d = dl + 1; d < 3; d++)   // a memory read of a ghost cell a later pass rewrites
                if (sg[d] != 0 && filled(b, d, sg[d])) race = true;
        };
        for (int b = H.lstart[L]; b < H.lstart[L + 1] && !race; b++)
            for (int sz = -1; sz <= 1; sz++)
                for (int sy = -1; sy <= 1; sy++)
                    for (int sx = -1; sx <= 1; sx++)
                        if (sx || sy || sz) walk(walk, b, {sx, sy, sz}, 2);
        return !race;
    }
    template <class TT, int N>
    void ghost_level_launch(int L, TT *u, bool cubic, int sel) {
        const int sweep = ghost_sweep_ctas<N>(cnt(L)), ngen = gCnt[L][sel + 1];
        const int ctas = sweep + ghost_general_ctas<N>(ngen);
        if (ctas == 0) return;
        launch_pdl(k_ghost_level<TT, N>, (unsigned)ctas, 256, 0, u, (const int32_t *)d_kind26[sel + 1],
                   (const GItem *)(d_gitems + gOff[L][sel + 1]), ngen, H.lstart[L], cnt(L), sweep,
                   (const GFace *)d_gface, (const int8_t *)d_oct, sel, cubic ? 1 : 0);
        ++launches;
    }
    // one fill of level L: k_ghost_level where exact, else the three passes
    template <class TT>
    void ghost_fill_level(int L, int f, TT *u, bool cubic, int sel) {
        const int n = nf[f];
        if (sel == 1 && L <= 0) return;
        const int mode = tune.get(kKnobGhostFill, (int)sizeof(TT), n, L, sel, 0);   // default: three passes
        const bool one = ghostForce >= 0 ? ghostForce == 1 : mode == 1;
        if (one && ghostMerge[L][sel + 1] && (n == 2 || n == 4 || n == 8 || n == 16)) {
            SFM_WITH_N(n, (ghost_level_launch<TT, N>(L, u, cubic, sel)), (void)0)
            return;
        }
        for (int dir = 0; dir < 3; dir++) ghost_pass(L, f, dir, u, cubic, sel);
    }

    // -----------------------------------------------------------------
    // ghost cells, convergence, boundary (any element type)
    template <class TT>
    void ghostcell_fix(int f, TT *u, bool cubic) {
        for (int L = 0; L < H.nlev; L++) ghost_fill_level(L, f, u, cubic, -1);
    }
    template <class TT, int N, int W>
    void ghost_pass_launch_w(TT *u, int64_t o, int64_t n0, int64_t sp, int64_t n1, int dir, bool cubic) {
        launch_pdl(k_ghost_faces<TT, N, W>,
                   (unsigned)(ghost_copy_ctas<N>((int)n0, W) +
                              (n1 + 256 / ghost_lanes<N>() - 1) / (256 / ghost_lanes<N>())),
                   256, 0, u, d_faces + o, (int)n0, d_faces + sp, (int)n1, dir, cubic ? 1 : 0);
    }
    template <class TT, int N>
    void ghost_pass_launch(TT *u, int64_t o, int64_t n0, int64_t sp, int64_t n1, int dir, bool cubic, bool aligned) {
        constexpr int WY = ghost_vec<TT, N>(1), WZ = ghost_vec<TT, N>(2);
        if (aligned && dir == 1) return ghost_pass_launch_w<TT, N, WY>(u, o, n0, sp, n1, dir, cubic);
        if (aligned && dir == 2) return ghost_pass_launch_w<TT, N, WZ>(u, o, n0, sp, n1, dir, cubic);
        ghost_pass_launch_w<TT, N, 1>(u, o, n0, sp, n1, dir, cubic);
    }
    template <class TT>
    void ghost_pass(int L, int f, int dir, TT *u, bool cubic, int sel = -1) {   // parentlev/samelev of (L, dir)
        const int k = L * 3 + dir;
        const int64_t o = faceOff[k], sp = faceSplit[k], c = faceOff[k + 1] - o;
        const int64_t n0 = sel != 1 ? sp - o : 0, n1 = sel != 0 ? faceOff[k + 1] - sp : 0;
        if (n0 + n1 <= 0) return;
        int GT = nf[f] + 2;
        const int n = nf[f];
        if ((n == 2 || n == 4 || n == 8 || n == 16) && n0 * GT * GT <= INT32_MAX) {
            // whole-vector copies of y rows and z planes need a 16-byte aligned field
            const bool aligned = ((uintptr_t)u & 15) == 0;
            SFM_WITH_N(n, (ghost_pass_launch<TT, N>(u, o, n0, sp, n1, dir, cubic, aligned), ++launches), (void)0)
            return;
        }
        run(OpGhostPass<TT>{u, d_faces + o, nf[f], Gf[f], Vf[f], dir, cubic ? 1 : 0, sel}, c * GT * GT);
    }
    template <class TT>
    void converge_c2p_lev(int Lc, int f, TT *u, bool cubic) {
        int Lf = Lc + 1, h = nf[f] / 2;
        SFM_WITH_N(nf[f],
                   (launch_pdl(k_converge_tiled<TT, N>, (unsigned)((cnt(Lf) + Tile<N>::BPC - 1) / Tile<N>::BPC), 256,
                               0, u, d_parent, d_oct, H.lstart[Lf], cnt(Lf), cubic ? 1 : 0),
                    ++launches),
                   run(OpConverge<TT>{u, d_parent, d_oct, H.lstart[Lf], nf[f], Gf[f], Vf[f], cubic ? 1 : 0},
                       (int64_t)cnt(Lf) * h * h * h))
    }
    template <class TT>
    void converge_c2p(int f, TT *u, bool cubic = false) {
        for (int Lc = H.nlev - 2; Lc >= 0; Lc--) converge_c2p_lev(Lc, f, u, cubic);
    }
    template <class TT>
    void boundary_fill0(int f, TT *u) {   // all blocks
        int64_t c = tfLOff[H.nlev];
        int GT = nf[f] + 2;
        run(OpFill0Faces<TT>{u, d_tfL, nf[f], Gf[f], Vf[f]}, c * GT * GT);
    }
    template <class TT>
    void boundary_fill0_level(int L, int f, TT *u) {
        int64_t o = tfLOff[L], c = tfLOff[L + 1] - o;
        int GT = nf[f] + 2;
        run(OpFill0Faces<TT>{u, d_tfL + o, nf[f], Gf[f], Vf[f]}, c * GT * GT);
    }
    template <class TT>
    void boundary_extrap(int f, TT *u) {   // all blocks, directions in order
        int GT = nf[f] + 2;
        for (int dir = 0; dir < 3; dir++) {
            int64_t o = tfDLOff[dir * H.nlev], c = tfDLOff[(dir + 1) * H.nlev] - o;
            run(OpExtrapFaces<TT>{u, d_tfDL + o, nf[f], Gf[f], Vf[f]}, c * GT * GT);
        }
    }
    template <class TT>
    void boundary_extrap_level(int L, int f, TT *u) {
        int GT = nf[f] + 2;
        for (int dir = 0; dir < 3; dir++) {
            int64_t o = tfDLOff[dir * H.nlev + L], c = tfDLOff[dir * H.nlev + L + 1] - o;
            run(OpExtrapFaces<TT>{u, d_tfDL + o, nf[f], Gf[f], Vf[f]}, c * GT * GT);
        }
    }
    template <class TT>
    void reflux(int f, const TT *u) {
        int h = nf[f] / 2;
        run(OpReflux<TT>{u, d_reflux, rbuf[f], d_h0, d_level, f, nf[f], Gf[f], Vf[f]}, (int64_t)nReflux * h * h);
    }
    // fmg_boundary_u / vmg_boundary_u: the z-mirror plane of the blocks of
    // AMR level L (or of all levels) touching the box's z-min face
    // (fmg_boundary_phys_zmirror.F90:55-80); the periodic and sphere
    // modules' hooks are no-ops
    template <class TT>
    void vmg_boundary_u(int L, int f, TT *u) {
        if (P.bc != SFM_BC_ZMIRROR || L < 0) return;
        const int64_t o = zminOff[L], c = zminOff[L + 1] - o;
        if (c > 0) run(OpMirrorZ<TT>{u, d_zmin + o, Gf[f], Vf[f]}, c * Gf[f] * Gf[f]);
    }
    template <class TT>
    void fmg_boundary_u(int f, TT *u) {   // every level in one launch (the blocks are independent)
        if (P.bc != SFM_BC_ZMIRROR) return;
        const int64_t c = zminOff[H.nlev];
        if (c > 0) run(OpMirrorZ<TT>{u, d_zmin, Gf[f], Vf[f]}, c * Gf[f] * Gf[f]);
    }
    // fmg_poisson_flux (fmg_poisson.F90:53-124)
    template <class TT>
    void poisson_flux(int f, TT *u, bool bf0) {
        if (FmgLevel_fill0 != f) {
            converge_c2p(f, u);
            fmg_boundary_u(f, u);
            ghostcell_fix(f, u, false);
            if (bf0) boundary_fill0(f, u);
            fmg_boundary_u(f, u);
        }
        FmgLevel_fill0 = Undef;
        reflux(f, u);
    }

    // -----------------------------------------------------------------
    // fmg level operations on the inner fields
    void relax(int f, T *u, T *rhs, bool bf0, int slot) {   // fmg_poisson_relax
        cudaMemsetAsync(d_max + slot, 0, sizeof(unsigned long long), st_);
        // the mixed schedule may sweep both colours in one launch (one ghost
        // refresh per sweep instead of one per colour)
        const bool fused = fused_at(f);
        for (int ipass = 1; ipass <= (fused ? 1 : 2); ipass++) {
            poisson_flux(f, u, bf0);
            const bool prof = f == 0 && profNext < (int)profEv.size() / 2;
            if (prof) prof_mark(2 * profNext);
            relax_launch(u, rhs, d_leaves, nLeaves, d_rslot, rbuf[f], f, ipass, d_max + slot, fused ? local_sweeps() : 0);
            if (prof) prof_mark(2 * profNext++ + 1);
        }
    }
    // both colours per launch at fmg level f: a mixed-path schedule choice
    // (fused_sweeps bit 0 for fmg_lin's sweeps, bit 1 for vmg_fas's), on
    // block edges the tiled and bulk-copy smoothers serve
    bool fused_at(int f, int bit = 1) const {
        if (sizeof(T) != 4 || serialRelax || !(sched(kKnobFusedSweep, 0) & bit)) return false;
        bool ok = false;
        SFM_WITH_N(nf[f], ok = N > 0, ok = false)
        return ok;
    }
    // full sweeps per fused launch (local_sweeps: 1, or 2 or 3 on the staged
    // block between ghost refreshes)
    int local_sweeps() const { return sched(kKnobLocalSweeps, 1); }
    // persistent grid of k_relax_bulk<T, N> (N >= 4): every SM filled to the
    // kernel's occupancy; computed once, at set-up, outside stream capture
    // the bulk pipeline serves blocks of 4^3 and up whose stages fit in 220 KB
    // (on 2^3 blocks it measured slower than k_relax_tiled)
    template <int N>
    static constexpr bool bulk_ok() { return N >= 4 && BulkPlan<T, N>::SMEM <= 220 * 1024; }
    // CTA sizes of the bulk-copy smoother: warp 0 produces, the rest
    // consume; 288 and 544 give 8 and 16 consumer warps, which divide a
    // colour's 256 cells (8^3 blocks, or eight 4^3 blocks) or 2048 cells
    // (16^3) evenly, where 256 and 512 leave a last partial round
    static constexpr int kRelaxNT[4] = {256, 288, 512, 544};
    template <int NT>
    static constexpr int nt_index() { return NT == 256 ? 0 : (NT == 288 ? 1 : (NT == 512 ? 2 : 3)); }
    template <int N, int NT, int SW>
    int bulk_grid() {
        if constexpr (!bulk_ok<N>()) {
            return 0;
        } else {
            constexpr int li = N >= 16 ? 4 : (N >= 8 ? 3 : 2);   // log2(N), capped
            constexpr int ti = nt_index<NT>();
            if (!bulkGrid[li][ti][SW]) {
                const int smem = BulkPlan<T, N>::SMEM;
                // opt in whatever the size: static and dynamic shared memory together may pass 48 KB
                cudaFuncSetAttribute(k_relax_bulk<T, N, NT, SW>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
                int per = 0;
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_relax_bulk<T, N, NT, SW>, NT, smem) !=
                        cudaSuccess ||
                    per < 1) {
                    cudaGetLastError();
                    per = 1;
                }
                bulkGrid[li][ti][SW] = nSM * per;
            }
            return bulkGrid[li][ti][SW];
        }
    }
    template <int N, int SW>
    void bulk_grids_of() {
        (void)bulk_grid<N, 256, SW>();
        (void)bulk_grid<N, 288, SW>();
        (void)bulk_grid<N, 512, SW>();
        (void)bulk_grid<N, 544, SW>();
    }
    template <int N>
    void bulk_grids() {   // every variant a solve may launch
        bulk_grids_of<N, 0>();
        if constexpr (sizeof(T) == 4) {
            bulk_grids_of<N, 1>();
            bulk_grids_of<N, 2>();
            bulk_grids_of<N, 3>();
        }
    }
    template <int N, int NT, int SW>
    void relax_bulk_launch(T *u, const T *rhs, const int32_t *blocks, int nblk, const int32_t *rslot, const double *rb,
                           int f, int ipass, unsigned long long *out) {
        launch_pdl(k_relax_bulk<T, N, NT, SW>,
                   (unsigned)std::min((nblk + Tile<N>::BPC - 1) / Tile<N>::BPC, bulk_grid<N, NT, SW>()), NT,
                   BulkPlan<T, N>::SMEM, u, rhs, blocks, nblk, d_h0, d_level, rslot, rb, f, ipass, out, d_err, waitPolls);
    }
    template <int N, int SW>
    void relax_bulk_nt(int nt, T *u, const T *rhs, const int32_t *blocks, int nblk, const int32_t *rslot,
                       const double *rb, int f, int ipass, unsigned long long *out) {
        switch (nt) {
            case 288: relax_bulk_launch<N, 288, SW>(u, rhs, blocks, nblk, rslot, rb, f, ipass, out); break;
            case 512: relax_bulk_launch<N, 512, SW>(u, rhs, blocks, nblk, rslot, rb, f, ipass, out); break;
            case 544: relax_bulk_launch<N, 544, SW>(u, rhs, blocks, nblk, rslot, rb, f, ipass, out); break;
            default: relax_bulk_launch<N, 256, SW>(u, rhs, blocks, nblk, rslot, rb, f, ipass, out); break;
        }
    }
    // CTA size of the bulk smoother at block edge n, two-launch sweep (tune
    // key kind -1) or fused sweeps (kind 1)
    int relax_nt(int n, bool fused) const {
        return tune.get(kKnobRelaxThreads, (int)sizeof(T), n, -1, fused ? 1 : -1, n >= 16 ? 512 : 256);
    }
    template <int N>
    void relax_dispatch(T *u, const T *rhs, const int32_t *blocks, int nblk, const int32_t *rslot, const double *rb,
                        int f, int ipass, unsigned long long *out, int sw) {
        if constexpr (bulk_ok<N>()) {
            const int nt = relax_nt(N, sw > 0);
            if constexpr (sizeof(T) == 4) {   // the FP64 path always runs the reference's two colour launches
                if (sw == 1) return relax_bulk_nt<N, 1>(nt, u, rhs, blocks, nblk, rslot, rb, f, ipass, out);
                if (sw == 2) return relax_bulk_nt<N, 2>(nt, u, rhs, blocks, nblk, rslot, rb, f, ipass, out);
                if (sw == 3) return relax_bulk_nt<N, 3>(nt, u, rhs, blocks, nblk, rslot, rb, f, ipass, out);
            }
            relax_bulk_nt<N, 0>(nt, u, rhs, blocks, nblk, rslot, rb, f, ipass, out);
        } else {
            launch_pdl(k_relax_tiled<T, N>, (unsigned)std::min((nblk + Tile<N>::BPC - 1) / Tile<N>::BPC, persistGrid),
                       256, 0, u, rhs, blocks, nblk, d_h0, d_level, rslot, rb, f, ipass, sizeof(T) == 4 ? sw : 0,
                       out);
        }
    }
    // one colour (ipass 1 or 2) over the listed blocks, or sw > 0 full
    // sweeps in one launch (fused_at decides; never on the per-element path)
    void relax_launch(T *u, const T *rhs, const int32_t *blocks, int nblk, const int32_t *rslot, const double *rb,
                      int f, int ipass, unsigned long long *out, int sw = 0) {
        const int n = nf[f];
        if (nblk <= 0) return;
        if (serialRelax) {   // race check: the same cells in a single-threaded sweep's order
            const int per = n * n * n / 2;
            launch_pdl(k_serial_blocks<OpRelax<T, T>>, (unsigned)((nblk + 127) / 128), 128, 0,
                       OpRelax<T, T>{u, rhs, blocks, d_h0, d_level, rslot, rb, f, n, Gf[f], Vf[f], ipass}, nblk, per, out);
            ++launches;
            return;
        }
        SFM_WITH_N(n, (relax_dispatch<N>(u, rhs, blocks, nblk, rslot, rb, f, ipass, out, sw), ++launches),
                   runMax(OpRelax<T, T>{u, rhs, blocks, d_h0, d_level, rslot, rb, f, n, Gf[f], Vf[f], ipass},
                          (int64_t)nblk * n * n * n / 2, out))
    }
    int check_err() {
        int e = 0;
        if (cudaMemcpy(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return SFM_ECUDA;
        if (e) { last_error = "a bulk-copy wait in the smoother gave up"; return SFM_ETIMEOUT; }
        return SFM_OK;
    }
    // Smoother timing (P.profile): an event pair around every level-0 colour
    // sweep of an outer iteration.  Inside stream capture the records become
    // event nodes of the iteration's graph (cudaEventRecordExternal), so the
    // timed solve keeps its graphs; the pairs are read after every iteration
    // (its residual read-back has synchronised the stream).
    static constexpr int kProfPairs = 64;
    std::vector<cudaEvent_t> profEv;   // 2 kProfPairs events, created at the first profiled solve
    int profNext = 0;                  // next pair while an iteration's launches are issued
    int profPairs = 0;                 // pairs one outer iteration records (kept with its graph)
    double profMs = 0.0;
    int64_t profN = 0;
    void prof_init() {
        profMs = 0.0;
        profN = 0;
        if (!P.profile || !profEv.empty()) return;
        profEv.assign(2 * kProfPairs, nullptr);
        for (auto &e : profEv)
            if (cudaEventCreate(&e) != cudaSuccess) {
                cudaGetLastError();
                e = nullptr;
            }
        for (auto e : profEv)
            if (!e) {   // no timing rather than a partial pool
                prof_release();
                break;
            }
    }
    void prof_release() {
        for (auto e : profEv)
            if (e) cudaEventDestroy(e);
        profEv.clear();
    }
    void prof_mark(int q) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(st_, &cs);
        cudaEventRecordWithFlags(profEv[q], st_,
                                 cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault);
    }
    void prof_iteration() {   // after an outer iteration's stream work has completed
        for (int q = 0; q < profPairs; q++) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, profEv[2 * q], profEv[2 * q + 1]) == cudaSuccess) {
                profMs += t;
                profN++;
            } else {
                cudaGetLastError();
            }
        }
    }
    void prof_collect(sfm_stats *stats) {
        if (stats) {
            stats->smoother_ms = profMs;
            stats->smoother_launches = profN;
            stats->smoother_cells = profN * nLeaves * H.NI * H.NI * H.NI;
            stats->smoother_colours = fused_at(0) ? 2 * local_sweeps() : 1;
        }
        profMs = 0.0;
        profN = 0;
    }
    template <class TU, class TR, class TO>
    void resid(int f, TO *res, TU *u, const TR *rhs, bool bf0) {   // fmg_poisson_resid
        poisson_flux(f, u, bf0);
        const int n = nf[f];
        if (n == 8) {   // blocks per CTA from the tuning table (default 2)
            const int bpc = tune.get(kKnobResidBpc, (int)sizeof(TU), 8, -1, -1, resid_bpc<8>());
            auto go = [&](auto kern, int b) {
                launch_pdl(kern, (unsigned)((nLeaves + b - 1) / b), 256, 0, res, u, rhs, d_leaves, nLeaves, d_h0, d_level,
                           d_rslot, rbuf[f], f);
            };
            if (bpc == 1) go(k_resid_tiled<TU, TR, TO, 8, 1>, 1);
            else if (bpc == 4) go(k_resid_tiled<TU, TR, TO, 8, 4>, 4);
            else go(k_resid_tiled<TU, TR, TO, 8, 2>, 2);
            ++launches;
            return;
        }
        SFM_WITH_N(n,
                   (launch_pdl(k_resid_tiled<TU, TR, TO, N>, (unsigned)((nLeaves + resid_bpc<N>() - 1) / resid_bpc<N>()),
                               256, 0, res, u, rhs, d_leaves, nLeaves, d_h0, d_level, d_rslot, rbuf[f], f),
                    ++launches),
                   run(OpResid<TU, TR, TO>{res, u, rhs, d_leaves, d_h0, d_level, d_rslot, rbuf[f], f, n, Gf[f], Vf[f]},
                       (int64_t)nLeaves * n * n * n))
    }
    void fmg_rstrct(int f, T *uc, const T *uf) {
        int nc = nf[f];
        run(OpRstrct<T, T>{uc, uf, d_leaves, nc, Gf[f], Gf[f - 1], Vf[f], Vf[f - 1]}, (int64_t)nLeaves * nc * nc * nc);
    }
    // element-wise over nblk whole listed blocks (k_blocks)
    template <class Op>
    void runB(const Op &op, int64_t nblk) {
        if (nblk <= 0) return;
        constexpr int W = Op::VW;
        if (op.V % W == 0 && op.aligned()) {   // whole vectors
            const int bpc = std::max(1, 256 / (int)(op.V / W));
            const int64_t g = std::min<int64_t>((nblk + bpc - 1) / bpc, (int64_t)nSM * 16);
            launch_pdl(k_blocks_vec<Op, W>, (unsigned)g, 256, 0, op, (int)nblk, bpc);
        } else {
            const int bpc = std::max(1, 256 / (int)op.V);
            const int64_t g = std::min<int64_t>((nblk + bpc - 1) / bpc, (int64_t)nSM * 16);
            launch_pdl(k_blocks<Op>, (unsigned)g, 256, 0, op, (int)nblk, bpc);
        }
        ++launches;
    }
    void fill0(int f, T *u) { runB(OpZero<T>{u, d_leaves, Vf[f]}, nLeaves); }
    template <class TO, class TI>
    void copy(int f, TO *o, const TI *a, bool noskip) {
        runB(OpCopy<TO, TI>{o, a, noskip ? d_all : d_leaves, Vf[f]}, noskip ? H.nb : nLeaves);
    }
    template <class TA, class TD>
    void add(int f, TA *a, const TD *d) { runB(OpAdd<TA, TD>{a, d, d_leaves, Vf[f]}, nLeaves); }

    // fmg_interp (fmg.F90:786-822)
    void fmg_interp(int f, T *uf, T *uc, bool cubic) {
        int lc = f + 1;
        converge_c2p(lc, uc, cubic);
        fmg_boundary_u(lc, uc);
        ghostcell_fix(lc, uc, cubic);
        boundary_extrap(lc, uc);
        fmg_boundary_u(lc, uc);
        const int n = nf[f];
        SFM_WITH_N(n,
                   (launch_pdl(k_interp_tiled<T, N>, (unsigned)((nLeaves + interp_bpc<N>() - 1) / interp_bpc<N>()), 256, 0, uf,
                               uc, d_leaves, nLeaves, cubic ? 1 : 0),
                    ++launches),
                   run(OpInterp<T>{uf, uc, d_leaves, n, Gf[f], Gf[lc], Vf[f], Vf[lc], cubic ? 1 : 0},
                       (int64_t)nLeaves * n * n * n))
        boundary_fill0(lc, uc);
        boundary_fill0(f, uf);
        fmg_boundary_u(lc, uc);
        fmg_boundary_u(f, uf);
    }

    // fmg_lin (fmg.F90:270-377)
    void fmg_lin() {
        nvtxRangePushA("sfm fmg_lin");
        const int FMax = H.FMax;
        for (int f = 1; f <= FMax; f++) fmg_rstrct(f, RHO[f], RHO[f - 1]);
        fill0(FMax, U[FMax]);
        vmg_fas(false);
        for (int f = FMax - 1; f >= 0; f--) {
            fmg_interp(f, U[f], U[f + 1], true);
            copy(f, RHS[f], RHO[f], false);
            const int ncycle = sched(kKnobFmgCycles, 2), nsweep = sched(kKnobFmgSweeps, 2);
            for (int jc = 1; jc <= ncycle; jc++) {
                for (int v = f; v <= FMax - 1; v++) {
                    for (int q = 0; q < nsweep; q++) relax(v, U[v], RHS[v], true, 0);
                    resid(v, RES[v], U[v], RHS[v], true);
                    fmg_rstrct(v + 1, RHS[v + 1], RES[v]);
                    fill0(v + 1, U[v + 1]);
                    FmgLevel_fill0 = v + 1;
                }
                vmg_fas(true);
                for (int v = FMax - 1; v >= f; v--) {
                    fmg_interp(v, RES[v], U[v + 1], false);   // fmg_addint
                    add(v, U[v], RES[v]);
                    for (int q = 0; q < nsweep; q++) relax(v, U[v], RHS[v], true, 0);
                }
            }
        }
        converge_c2p(0, U[0]);
        nvtxRangePop();
    }

    // -----------------------------------------------------------------
    // vmg (vmg.F90) at fmg level FMax
    // (vmg_poisson_flux mirrors once more after vmg_ghostcell,
    // vmg_poisson.F90:73-74: the plane it copies is unchanged since the
    // mirror at the end of vmg_ghostcell, so that copy is left out)
    void vmg_ghostcell(int L, T *u) {   // vmg.F90:729-743
        const int F = H.FMax;
        vmg_boundary_u(L, F, u);
        ghost_fill_level(L, F, u, false, 0);   // same-level faces, x then y then z
        boundary_fill0_level(L, F, u);
        vmg_boundary_u(L, F, u);
    }
    void vmg_gridboundary(int L, T *u) {   // vmg.F90:710-725
        const int F = H.FMax;
        vmg_boundary_u(L - 1, F, u);
        ghost_fill_level(L, F, u, false, 1);   // coarse-fine faces, x then y then z
        boundary_fill0_level(L, F, u);
        vmg_boundary_u(L, F, u);
    }
    void vmg_relax(int L, T *u, const T *rhs) {   // vmg_poisson_relax (vmg_poisson.F90:98-145)
        const int F = H.FMax;
        const bool fused = fused_at(F, 2);
        for (int ipass = 1; ipass <= (fused ? 1 : 2); ipass++) {
            vmg_ghostcell(L, u);
            relax_launch(u, rhs, d_all + H.lstart[L], cnt(L), nullptr, nullptr, F, ipass, d_max + 1,
                         fused ? local_sweeps() : 0);
        }
    }
    void vmg_rstrct(int Lc, T *u, bool cubic) {
        const int F = H.FMax;
        if (cubic) ghost_fill_level(Lc + 1, F, u, true, -1);   // per direction: coarse-fine, then same level
        converge_c2p_lev(Lc, F, u, cubic);
    }
    void vmg_copy_level(int L, T *o, const T *a) {
        const int F = H.FMax;
        runB(OpCopy<T, T>{o, a, d_all + H.lstart[L], Vf[F]}, cnt(L));
    }
    void vmg_tau(int L) {   // vmg_poisson_tau + vmg_tau_crop, tau in RES
        const int F = H.FMax, n = nf[F];
        int Lf = L + 1;
        if (Lf > H.nlev - 1) return;
        vmg_ghostcell(Lf, U[F]);
        run(OpTauFine<T>{RES[F], U[F], H.lstart[Lf], n, Gf[F], Vf[F], (T)(1.0 / hlev(H.h0.data(), Lf, F))},
            (int64_t)cnt(Lf) * Vf[F]);
        converge_c2p_lev(L, F, RES[F], false);
        vmg_ghostcell(L, U[F]);
        int64_t wc = wcOff[L + 1] - wcOff[L];
        run(OpTauParent<T>{RES[F], U[F], d_withChild + wcOff[L], n, Gf[F], Vf[F], (T)(1.0 / hlev(H.h0.data(), L, F))},
            wc * n * n * n);
        int64_t co = cropOff[Lf], cc = cropOff[Lf + 1] - co;
        int GT = n + 2;
        run(OpTauCrop<T>{RES[F], d_crop + co, d_parent, n, Gf[F], Vf[F]}, cc * GT * GT);
    }
    void vmg_interp(int Lf, T *uf, T *uc) {   // vmg_interp (vmg.F90:592-601)
        const int F = H.FMax, n = nf[F];
        int Lc = Lf - 1;
        vmg_ghostcell(Lc, uc);
        boundary_extrap_level(Lc, F, uc);
        vmg_boundary_u(Lc, F, uc);
        run(OpP2C<T>{uf, uc, d_parent, d_oct, H.lstart[Lf], n, Gf[F], Vf[F]}, (int64_t)cnt(Lf) * n * n * n);
        boundary_fill0_level(Lc, F, uc);
        vmg_boundary_u(Lc, F, uc);
    }
    void vmg_zeroAverage(T *a) {
        const int F = H.FMax, n = nf[F];
        run(OpBlockSum<T>{a, d_all, d_psum, n, Gf[F], Vf[F]}, (int64_t)cnt(0));
        launch_pdl(k_ave_combine_w, 1, 1024, 0, d_psum, cnt(0), n, d_scal + 1);
        ++launches;
        run(OpSubScalarInterior<T>{a, d_scal + 1, 0, n, Gf[F], Vf[F]}, (int64_t)cnt(0) * n * n * n);
    }
    void vmg_slvsml(T *u, T *rhs) {
        if (!useSerialMg) {
            for (int q = 0; q < 10; q++) vmg_relax(0, u, rhs);
            return;
        }
        const int F = H.FMax;
        int64_t N3 = (int64_t)NBc * NBc * NBc;
        run(OpMgGather<T>{mg.SRC, mg.PSI, rhs, u, d_baseIdx, H.ngb[0], H.ngb[1], nf[F], Gf[F], NBc, Vf[F]}, N3);
        mg_launch(tune.get(kKnobBaseCtas, (int)sizeof(T), NBc, -1, -1, 1),
                  tune.get(kKnobBaseWide, (int)sizeof(T), NBc, -1, -1, 16));
        run(OpMgScatter<T>{u, mg.PSI, d_baseIdx, H.ngb[0], H.ngb[1], nf[F], Gf[F], NBc, Vf[F]}, N3);
    }
    // vmg_fas (vmg.F90:116-243); jrho = IRHS when copy_rhs (second and later calls)
    void vmg_fas(bool copy_rhs) {
        nvtxRangePushA("sfm vmg_fas");
        const int F = H.FMax, nlev = H.nlev;
        // the level lists are consecutive ranges of d_all: the per-level
        // copies of vmg_fas are one launch over all blocks
        if (copy_rhs) runB(OpCopy<T, T>{RHO[F], RHS[F], d_all, Vf[F]}, H.nb);
        converge_c2p(F, U[F]);
        converge_c2p(F, RHO[F]);
        boundary_fill0(F, U[F]);
        fmg_boundary_u(F, U[F]);
        runB(OpCopy<T, T>{RHS[F], RHO[F], d_all, Vf[F]}, H.nb);
        const int nvs = sched(kKnobVmgSweeps, 2);
        for (int v = nlev - 1; v >= 1; v--) {
            vmg_gridboundary(v, U[F]);
            for (int q = 0; q < nvs; q++) vmg_relax(v, U[F], RHS[F]);
            vmg_rstrct(v - 1, U[F], true);
            vmg_copy_level(v - 1, RUF, U[F]);
            vmg_rstrct(v - 1, RHS[F], false);
            vmg_tau(v - 1);
            int64_t wc = wcOff[v] - wcOff[v - 1];
            runB(OpAdd<T, T>{RHS[F], RES[F], d_withChild + wcOff[v - 1], Vf[F]}, wc);
        }
        if (P.zero_mean) vmg_zeroAverage(RHS[F]);
        vmg_slvsml(U[F], RHS[F]);
        for (int v = 1; v <= nlev - 1; v++) {
            runB(OpSub<T>{RES[F], U[F], RUF, d_all + H.lstart[v - 1], Vf[F]}, cnt(v - 1));
            vmg_interp(v, RES[F], RES[F]);
            runB(OpAdd<T, T>{U[F], RES[F], d_all + H.lstart[v], Vf[F]}, cnt(v));
            vmg_gridboundary(v, U[F]);
            for (int q = 0; q < nvs; q++) vmg_relax(v, U[F], RHS[F]);
        }
        nvtxRangePop();
    }

    // -----------------------------------------------------------------
    // outer FP64 stages
    // sphere and z-mirror: mask SRC0, moments, multipole ghosts of PSI0
    // (fmg_boundary_phys_sphere.F90:81-354, fmg_boundary_phys_zmirror.F90:100-382)
    void boundary_physical_grid() {
        if (zperiodic()) return boundary_physical_grid_cyl();
        if (P.bc != SFM_BC_SPHERE && P.bc != SFM_BC_ZMIRROR && P.bc != SFM_BC_SPHERE_MHD_BE) return;
        const bool zm = P.bc == SFM_BC_ZMIRROR;
        const int n = H.NI;
        int bmin = H.baseIdx.front(), bmax = H.baseIdx.back();
        auto X = [&](int b, int d, int i) { return H.x0[3 * b + d] + (double)i * H.h0[H.level[b]]; };
        double xmin = X(bmin, 0, 0), ymin = X(bmin, 1, 0), zmin = X(bmin, 2, 0);
        double xmax = X(bmax, 0, n - 1), ymax = X(bmax, 1, n - 1), zmax = X(bmax, 2, n - 1);
        // the z-mirror box's z-min face is the mirror plane, not an edge of the sphere
        double rr = zm ? std::min(std::min(std::min(xmax, ymax), zmax), std::min(-xmin, -ymin))
                       : std::min(std::min(std::min(xmax, ymax), std::min(zmax, -xmin)), std::min(-ymin, -zmin));
        if (P.bc == SFM_BC_SPHERE_MHD_BE) rr = P.r_cloud;   // the cloud's radius (sphere_MHD_BE.F90:72)
        double rad2 = rr * rr;
        run(OpSphereMask{SRC0, d_x0, d_h0, d_level, n, Gf[0], Vf[0], rad2}, (int64_t)H.nb * Vf[0]);
        const int64_t ncell = (int64_t)cnt(0) * n * n * n;
        launch_pdl(k_moment_terms, (unsigned)std::min<int64_t>((ncell + 255) / 256, (int64_t)nSM * 8), 256, 0, SRC0,
                   d_x0, d_h0, n, Gf[0], Vf[0], cnt(0), P.lmax, d_part);
        launch_pdl(k_moments_ordered, 1, 32, 0, d_part, ncell, d_mom, zm ? 1 : 0, 1.0, 1.0);
        launches += 2;
        int GT = n + 2;
        run(OpSphereGhost{PSI0, d_tfL, d_mom, d_x0, d_h0, d_level, n, Gf[0], Vf[0], P.lmax}, tfLOff[H.nlev] * GT * GT);
    }

    // z-periodic cylinder and its density-masked variant
    // (fmg_boundary_phys_cyl_zperiodic.F90:97-232, ..._mask_zperiodic.F90):
    // mask SRC0, a00 = (sum of rho dv over the base-level cells, in the
    // reference's order) / zlen / (2 pi), ghost = a00 ln(r) on the x and y faces
    void boundary_physical_grid_cyl() {
        const int n = H.NI;
        int bmin = H.baseIdx.front(), bmax = H.baseIdx.back();
        auto X = [&](int b, int d, int i) { return H.x0[3 * b + d] + (double)i * H.h0[H.level[b]]; };
        double xmin = X(bmin, 0, 0), ymin = X(bmin, 1, 0), zmin = X(bmin, 2, 0);
        double xmax = X(bmax, 0, n - 1), ymax = X(bmax, 1, n - 1), zmax = X(bmax, 2, n - 1);
        const double zlen = zmax - zmin + H.h0[0];
        if (P.bc == SFM_BC_CYL_ZPERIODIC) {
            double rr = std::min(std::min(xmax, ymax), std::min(-xmin, -ymin));
            run(OpCylMask{SRC0, d_x0, d_h0, d_level, n, Gf[0], Vf[0], rr * rr}, (int64_t)H.nb * Vf[0]);
        } else {
            run(OpRhoMask{SRC0, P.rho_mask}, (int64_t)H.nb * Vf[0]);
        }
        const int64_t ncell = (int64_t)cnt(0) * n * n * n;
        launch_pdl(k_moment_terms, (unsigned)std::min<int64_t>((ncell + 255) / 256, (int64_t)nSM * 8), 256, 0, SRC0,
                   d_x0, d_h0, n, Gf[0], Vf[0], cnt(0), P.lmax, d_part);
        const double pi2 = 2.0 * (4.0 * std::atan(1.0));   // Pi2 (parameter.F90:14-15)
        launch_pdl(k_moments_ordered, 1, 32, 0, d_part, ncell, d_mom, 2, zlen, pi2);
        launches += 2;
        int GT = n + 2;
        run(OpCylGhost{PSI0, d_tfL, d_cyllog, d_mom, n, Gf[0], Vf[0]}, tfLOff[H.nlev] * GT * GT);
    }

    double read_max(int slot) {
        unsigned long long v = 0;
        cudaMemcpyAsync(&v, d_max + slot, sizeof(v), cudaMemcpyDeviceToHost, st_);
        cudaStreamSynchronize(st_);
        double d;
        std::memcpy(&d, &v, sizeof(d));
        return d;
    }
    void h2absmax(const double *a, int slot) {
        const int n = nf[0];
        cudaMemsetAsync(d_max + slot, 0, sizeof(unsigned long long), st_);
        runMax(OpH2Abs<double>{a, d_leaves, d_h0, d_level, 0, n, Gf[0], Vf[0]}, (int64_t)nLeaves * n * n * n, d_max + slot);
    }

    int check(const char *where) {
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
        if (e != cudaSuccess) {
            last_error = std::string(where) + ": " + cudaGetErrorString(e);
            return SFM_ECUDA;
        }
        return SFM_OK;
    }

    // fmg_cycle (fmg.F90:134-233) on device arrays
    int solve(const double *rho, double *psi, double *g, sfm_stats *stats, cudaStream_t s, int stop_stage,
              double *dump) override {
        st_ = s ? s : own_;   // all work of this call is ordered on the caller's stream
        launches = 0;
        prof_init();
        const int nb = H.nb, gw = ioGw > 0 ? ioGw : P.ngh_io;
        cudaEventRecord(ev0, st_);
        // fresh, zero-filled arrays as fmg_alloc_arr gives (fmg_data.F90:393)
        for (auto &z : zeroList) cudaMemsetAsync(z.first, 0, z.second, st_);
        cudaMemsetAsync(d_bad, 0, sizeof(int), st_);
        FmgLevel_fill0 = Undef;
        // fmg_make_physvar
        run(OpPhysvar<double>{PHI0, RES0d, rho, psi, H.NI, Gf[0], gw, Vf[0], P.four_pi_G, d_bad}, (int64_t)nb * Vf[0]);
        if (P.zero_mean) {
            run(OpBlockSum<double>{RES0d, d_leaves, d_psum, H.NI, Gf[0], Vf[0]}, (int64_t)nLeaves);
            launch_pdl(k_mean_combine_w, 1, 1024, 0, d_psum, d_leaves, nLeaves, d_level, d_h0, H.NI, d_scal);
            ++launches;
            run(OpSubScalarAll<double>{RES0d, d_scal}, (int64_t)nb * Vf[0]);
        } else {
            cudaMemsetAsync(d_scal, 0, sizeof(double), st_);
        }
        copy(0, RHO[0], RES0d, true);   // IRHO(f0) as the reference holds it
        copy(0, U[0], PHI0, true);      // IU(f0)
        copy(0, PSI0, PHI0, false);     // fmg_copy(IPSI, IU)
        copy(0, SRC0, RES0d, false);    // fmg_copy(ISRC, IRHO)
        converge_c2p(0, SRC0);
        converge_c2p(0, PSI0);
        boundary_physical_grid();
        fmg_boundary_u(0, PSI0);
        h2absmax(SRC0, 2);
        int rc = check("setup");
        if (rc) return rc;
        int bad = 0;
        cudaMemcpy(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost);
        if (bad) return SFM_ENONFINITE;
        double resh2max = read_max(2), rhoave = 0.0;
        cudaMemcpy(&rhoave, d_scal, sizeof(double), cudaMemcpyDeviceToHost);
        if (stop_stage == 1) return dumpd(SRC0, dump);
        if (stats) { std::memset(stats, 0, sizeof(*stats)); stats->resh2max = resh2max; stats->rho_mean = rhoave; }
        double ratio_prev = std::numeric_limits<double>::max();
        int nmax = P.max_outer;
        if (std::fabs(resh2max) <= std::numeric_limits<double>::min()) nmax = 0;
        bool conv = true, reached = (nmax == 0);
        int iters = 0;
        for (int it = 1; it <= nmax; it++) {
            if (stop_stage == 2 || stop_stage == 3) {
                resid<double, double, T>(0, RHO[0], PSI0, SRC0, false);
                if (stop_stage == 2) { rc = check("resid"); return rc ? rc : dumpT(RHO[0], dump); }
                fmg_lin();
                rc = check("fmg_lin");
                return rc ? rc : dumpT(U[0], dump);
            }
            outer_iteration();
            rc = check("outer");
            if (rc) return rc;
            iters = it;
            double ratio = read_max(0) / resh2max;
            prof_iteration();
            if (stats && it <= SFM_MAX_HISTORY) stats->ratio[it - 1] = ratio;
            if (ratio < P.rel_tol) { reached = true; break; }
            if (it == nmax) conv = false;
            if (P.stagnation_exit && ratio > ratio_prev * 0.5) conv = false;
            if (!conv) break;
            ratio_prev = ratio;
        }
        if (stop_stage == 4) return dumpd(PSI0, dump);
        copy(0, PHI0, PSI0, true);
        converge_c2p(0, PHI0);
        fmg_boundary_u(0, PHI0);
        poisson_flux(0, PHI0, false);
        if (g)
            run(OpPsi2g{g, PHI0, d_skip, d_level, d_h0, d_rslot, rbuf[0], H.NI, Gf[0], gCompact ? 0 : gw, Vf[0]},
                (int64_t)nb * H.NI * H.NI * H.NI);
        if (psi) run(OpRestore{psi, PHI0, H.NI, Gf[0], gw, Vf[0]}, (int64_t)nb * Vf[0]);
        cudaEventRecord(ev1, st_);
        double trr = 0.0;
        if (P.report_residual && resh2max > 0) {
            FmgLevel_fill0 = Undef;
            resid<double, double, double>(0, RES0d, PHI0, SRC0, false);
            h2absmax(RES0d, 3);
            trr = read_max(3) / resh2max;
        }
        rc = check("finish");
        if (rc == SFM_OK) rc = check_err();
        if (rc) return rc;
        if (stats) {
            stats->outer_iters = iters;
            stats->converged = (conv && reached) ? 1 : 0;
            stats->true_rel_residual = trr;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev0, ev1);
            stats->device_ms = ms;
            stats->kernel_launches = launches;
            stats->elem_bytes = (int32_t)sizeof(T);
        }
        prof_collect(stats);
        return (conv && reached) ? SFM_OK : SFM_ENOTCONVERGED;
    }
    // -----------------------------------------------------------------
    // adjoint of the converged solve (sfm_adjoint; device side in
    // sfm_adjoint.cuh).  FGMRES(m) on A^T lambda = dJ/dphi, right-
    // preconditioned with W M W^-1 (M one fmg_lin of this solver, W the cell
    // volumes: the conservative flux form makes W A nearly symmetric, so
    // A^T ~ W A W^-1), then the chain rule through the multipole boundary,
    // the mask and the mean removal back to rho.
    // -----------------------------------------------------------------
    bool adjReady = false;
    int adjM = 0, nAdjRefl = 0;
    AdjReflux *d_adjRefl = nullptr;
    int8_t *d_touch = nullptr;
    double *aG = nullptr, *aLam = nullptr, *aR = nullptr, *aW = nullptr, *aUB = nullptr, *aS = nullptr,
           *aIO = nullptr, *aPart = nullptr, *aBeta = nullptr, *aDot = nullptr;
    double *aF[3] = {nullptr, nullptr, nullptr};
    std::vector<double *> aV, aZ;

    int adj_init() {
        if (adjReady) return SFM_OK;
        std::vector<AdjReflux> ar;
        for (int L = 1; L < H.nlev; L++)
            for (int b = H.lstart[L]; b < H.lstart[L + 1]; b++)
                for (int dir = 0; dir < 3; dir++)
                    for (int lr = 0; lr < 2; lr++) {
                        const int f = lr + 2 * dir;
                        if (!H.parLev[6 * b + f]) continue;
                        AdjReflux it;
                        it.fine = b; it.coarse = H.nbrGid[6 * b + f]; it.dir = (int8_t)dir; it.lr = (int8_t)lr;
                        it.oa = H.oct[3 * b + tra(dir)]; it.ob = H.oct[3 * b + trb(dir)];
                        ar.push_back(it);
                    }
        nAdjRefl = (int)ar.size();
        d_adjRefl = mem.upload(ar);
        d_touch = mem.upload(H.touch);
        const size_t NV = (size_t)H.nb * Vf[0];
        const int gw = P.ngh_io;
        const size_t NIO = (size_t)H.nb * (size_t)(H.NI + 2 * gw) * (H.NI + 2 * gw) * (H.NI + 2 * gw);
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        const size_t per = NV * sizeof(double);
        const double avail = 0.8 * (double)fr - (double)NIO * sizeof(double);
        const long vecs = (long)(avail / (double)per) - 9;   // G, lambda, R, W, UB, 3 fluxes, S
        const long m = (vecs - 1) / 2;
        if (m < 2) return SFM_ENOMEM;
        adjM = (int)std::min<long>(m, 30);
        aG = mem.alloc<double>(NV); aLam = mem.alloc<double>(NV); aR = mem.alloc<double>(NV);
        aW = mem.alloc<double>(NV); aUB = mem.alloc<double>(NV); aS = mem.alloc<double>(NV);
        for (auto &f : aF) f = mem.alloc<double>(NV);
        for (int j = 0; j <= adjM; j++) aV.push_back(mem.alloc<double>(NV));
        for (int j = 0; j < adjM; j++) aZ.push_back(mem.alloc<double>(NV));
        aIO = mem.alloc<double>(NIO);
        aPart = mem.alloc<double>((size_t)std::max<int64_t>(tfLOff[H.nlev], 1) * 25);
        aBeta = mem.alloc<double>(32);
        aDot = mem.alloc<double>(8);
        if (mem.err != cudaSuccess) {
            last_error = cudaGetErrorString(mem.err);
            return mem.err == cudaErrorMemoryAllocation ? SFM_ENOMEM : SFM_ECUDA;
        }
        adjReady = true;
        return SFM_OK;
    }
    int64_t adj_nv() const { return (int64_t)H.nb * Vf[0]; }
    void adj_leaf_only(double *a) { run(OpLeafInterior{a, d_skip, nf[0], Gf[0], Vf[0]}, adj_nv()); }
    void adj_converge_T(double *a) {
        const int n = nf[0], h = n / 2;
        for (int Lc = 0; Lc <= H.nlev - 2; Lc++)
            run(OpConvergeT{a, d_parent, d_oct, H.lstart[Lc + 1], n, Gf[0], Vf[0]}, (int64_t)cnt(Lc + 1) * h * h * h);
    }
    // ordered sum over leaf interiors of a*b (of a when b is null)
    double adj_dot(const double *a, const double *b) {
        run(OpBlockDot{a, b, d_leaves, d_psum, nf[0], Gf[0], Vf[0]}, (int64_t)nLeaves);
        launch_pdl(k_sum_ordered, 1, 32, 0, d_psum, nLeaves, aDot);
        ++launches;
        double v = 0.0;
        cudaMemcpyAsync(&v, aDot, sizeof(double), cudaMemcpyDeviceToHost, st_);
        cudaStreamSynchronize(st_);
        return v;
    }
    // aUB = (residual pipeline)^T g: A^T g on leaf interiors, A_bc^T g on
    // the physical ghosts
    void adj_apply_AT(const double *g) {
        const int n = nf[0], G = Gf[0], GT = n + 2, h = n / 2;
        const int64_t V = Vf[0], NV = adj_nv();
        run(OpDivT{aF[0], aF[1], aF[2], g, d_skip, d_h0, d_level, n, G, V}, NV);
        run(OpRefluxT{aF[0], aF[1], aF[2], d_adjRefl, n, G, V}, (int64_t)nAdjRefl * h * h);
        run(OpFluxT{aUB, aF[0], aF[1], aF[2], d_skip, d_h0, d_level, n, G, V}, NV);
        for (int L = H.nlev - 1; L >= 0; L--)
            for (int dir = 2; dir >= 0; dir--) {
                const int64_t o = faceOff[L * 3 + dir], c = faceOff[L * 3 + dir + 1] - o;
                run(OpGhostT{aUB, d_faces + o, n, G, V, dir}, c * GT * GT);
            }
        adj_converge_T(aUB);
    }
    void adj_precond(const double *v, double *z) {
        const int64_t NV = adj_nv();
        run(OpPrecIn<T>{RHO[0], v, d_skip, d_h0, d_level, nf[0], Gf[0], Vf[0]}, NV);
        FmgLevel_fill0 = Undef;
        fmg_lin();
        run(OpPrecOut<T>{z, U[0], d_skip, d_h0, d_level, nf[0], Gf[0], Vf[0]}, NV);
    }
    void adj_copy(double *o, const double *a) {
        cudaMemcpyAsync(o, a, (size_t)adj_nv() * sizeof(double), cudaMemcpyDeviceToDevice, st_);
    }
    double sphere_rad2() const {
        const int n = H.NI;
        int bmin = H.baseIdx.front(), bmax = H.baseIdx.back();
        auto X = [&](int b, int d, int i) { return H.x0[3 * b + d] + (double)i * H.h0[H.level[b]]; };
        double xmin = X(bmin, 0, 0), ymin = X(bmin, 1, 0), zmin = X(bmin, 2, 0);
        double xmax = X(bmax, 0, n - 1), ymax = X(bmax, 1, n - 1), zmax = X(bmax, 2, n - 1);
        double rr = std::min(std::min(std::min(xmax, ymax), std::min(zmax, -xmin)), std::min(-ymin, -zmin));
        return rr * rr;
    }

    int adjoint(const double *dJdphi, double *dJdrho, sfm_stats *stats, cudaStream_t s) override {
        if (P.bc == SFM_BC_ZMIRROR || zperiodic() || P.bc == SFM_BC_SPHERE_MHD_BE) {
            // these boundaries' transposes are not built
            last_error = "sfm_adjoint: periodic and sphere boxes only";
            return SFM_EINVAL;
        }
        st_ = s ? s : own_;
        launches = 0;
        int rc = adj_init();
        if (rc) return rc;
        cudaEventRecord(ev0, st_);
        const int n = nf[0], G = Gf[0], gw = P.ngh_io;
        const int64_t V = Vf[0], NV = adj_nv();
        const int64_t NIO = (int64_t)H.nb * (n + 2 * gw) * (n + 2 * gw) * (n + 2 * gw);
        for (auto &z : zeroList) cudaMemsetAsync(z.first, 0, z.second, st_);   // fresh inner arrays
        cudaMemcpyAsync(aIO, dJdphi, (size_t)NIO * sizeof(double), cudaMemcpyHostToDevice, st_);
        run(OpAdjIn{aG, aIO, n, G, gw, V}, NV);
        adj_converge_T(aG);   // phi on covered blocks is the restriction of the leaves
        adj_leaf_only(aG);
        const double ncell = (double)nLeaves * n * n * n;
        if (P.bc == SFM_BC_PERIODIC) {   // A is singular (constants): keep g orthogonal to them
            const double mean = adj_dot(aG, nullptr) / ncell;
            run(OpAxpyLeafConst{aG, -mean, d_skip, n, G, V}, NV);
        }
        if (stats) std::memset(stats, 0, sizeof(*stats));
        const int m = adjM, maxit = std::max(1, P.max_outer);
        const double tol = P.rel_tol;
        const double gnorm = std::sqrt(adj_dot(aG, aG));
        cudaMemsetAsync(aLam, 0, (size_t)NV * sizeof(double), st_);
        adj_copy(aR, aG);
        double beta = gnorm, trr = 0.0;
        int iters = 0;
        bool reached = gnorm == 0.0;
        std::vector<double> Hm((size_t)(m + 1) * m), cs(m), sn(m), sv(m + 1), y;
        auto Hij = [&](int i, int j) -> double & { return Hm[(size_t)i * m + j]; };
        while (!reached && iters < maxit) {
            std::fill(Hm.begin(), Hm.end(), 0.0);
            std::fill(sv.begin(), sv.end(), 0.0);
            adj_copy(aV[0], aR);
            run(OpScale{aV[0], 1.0 / beta}, NV);
            sv[0] = beta;
            int jlast = -1;
            for (int j = 0; j < m && iters < maxit; j++) {
                adj_precond(aV[j], aZ[j]);
                adj_apply_AT(aZ[j]);
                adj_copy(aW, aUB);
                adj_leaf_only(aW);
                for (int i = 0; i <= j; i++) {
                    Hij(i, j) = adj_dot(aW, aV[i]);
                    run(OpAxpy{aW, aV[i], -Hij(i, j)}, NV);
                }
                Hij(j + 1, j) = std::sqrt(adj_dot(aW, aW));
                adj_copy(aV[j + 1], aW);
                if (Hij(j + 1, j) > 0.0) run(OpScale{aV[j + 1], 1.0 / Hij(j + 1, j)}, NV);
                for (int i = 0; i < j; i++) {
                    const double t = cs[i] * Hij(i, j) + sn[i] * Hij(i + 1, j);
                    Hij(i + 1, j) = -sn[i] * Hij(i, j) + cs[i] * Hij(i + 1, j);
                    Hij(i, j) = t;
                }
                const double den = std::hypot(Hij(j, j), Hij(j + 1, j));
                cs[j] = den > 0 ? Hij(j, j) / den : 1.0;
                sn[j] = den > 0 ? Hij(j + 1, j) / den : 0.0;
                Hij(j, j) = den;
                Hij(j + 1, j) = 0.0;
                sv[j + 1] = -sn[j] * sv[j];
                sv[j] = cs[j] * sv[j];
                iters++;
                jlast = j;
                const double rel = std::fabs(sv[j + 1]) / gnorm;
                if (stats && iters <= SFM_MAX_HISTORY) stats->ratio[iters - 1] = rel;
                if (rel < tol) break;
            }
            y.assign(jlast + 1, 0.0);
            for (int i = jlast; i >= 0; i--) {
                double t = sv[i];
                for (int k = i + 1; k <= jlast; k++) t -= Hij(i, k) * y[k];
                y[i] = t / Hij(i, i);
            }
            for (int i = 0; i <= jlast; i++) run(OpAxpy{aLam, aZ[i], y[i]}, NV);
            adj_apply_AT(aLam);
            run(OpSubArr{aR, aG, aUB}, NV);
            adj_leaf_only(aR);
            beta = std::sqrt(adj_dot(aR, aR));
            trr = gnorm > 0 ? beta / gnorm : 0.0;
            reached = trr < tol;
        }
        if (gnorm == 0.0) cudaMemsetAsync(aUB, 0, (size_t)NV * sizeof(double), st_);
        // aUB holds the transposed pipeline applied to lambda
        cudaMemsetAsync(aS, 0, (size_t)NV * sizeof(double), st_);
        double rad2 = -1.0;
        if (P.bc == SFM_BC_SPHERE) {
            rad2 = sphere_rad2();
            const int64_t nfaces = tfLOff[H.nlev];
            run(OpBcBeta{aUB, d_tfL, d_touch, d_x0, d_h0, d_level, aPart, n, G, V, P.lmax}, nfaces);
            launch_pdl(k_bc_beta_combine, 1, 32, 0, aPart, (int)nfaces, aBeta);
            ++launches;
            run(OpMomentT{aS, aBeta, d_x0, d_h0, H.lstart[0], n, G, V, rad2, P.lmax}, (int64_t)cnt(0) * n * n * n);
            adj_converge_T(aS);
        }
        run(OpAddMaskedLambda{aS, aLam, d_skip, d_x0, d_h0, d_level, n, G, V, rad2}, NV);
        double corr = 0.0;
        if (P.zero_mean) {
            double vol = 0.0;
            for (int b : leafList) {
                const double h = H.h0[H.level[b]];
                vol += (double)(n * n * n) * (h * h * h);
            }
            corr = adj_dot(aS, nullptr) / vol;
        }
        run(OpAdjOut{aIO, aS, d_skip, d_h0, d_level, n, G, gw, V, P.four_pi_G, corr}, NIO);
        cudaMemcpyAsync(dJdrho, aIO, (size_t)NIO * sizeof(double), cudaMemcpyDeviceToHost, st_);
        cudaEventRecord(ev1, st_);
        rc = check("adjoint");
        if (rc == SFM_OK) rc = check_err();
        if (rc) return rc;
        if (stats) {
            stats->outer_iters = iters;
            stats->converged = reached ? 1 : 0;
            stats->true_rel_residual = trr;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev0, ev1);
            stats->device_ms = ms;
            stats->kernel_launches = launches;
            stats->elem_bytes = (int32_t)sizeof(T);
        }
        return reached ? SFM_OK : SFM_ENOTCONVERGED;
    }

    int dumpd(const double *a, double *dump) {
        int rc = check("dump");
        if (rc) return rc;
        if (dump) cudaMemcpy(dump, a, (size_t)H.nb * Vf[0] * sizeof(double), cudaMemcpyDeviceToHost);
        return SFM_OK;
    }
    int dumpT(const T *a, double *dump) {
        if (!dump) return SFM_OK;
        std::vector<T> tmp((size_t)H.nb * Vf[0]);
        cudaMemcpy(tmp.data(), a, tmp.size() * sizeof(T), cudaMemcpyDeviceToHost);
        for (size_t i = 0; i < tmp.size(); i++) dump[i] = (double)tmp[i];
        return SFM_OK;
    }
};

}  // namespace sfm

// =============================================================================
// C ABI
// =============================================================================
struct sfm_ctx {
    sfm::SolverBase *s = nullptr;
    sfm_params p;
    int device = 0, nb = 0, ni = 0, ngh = 0;
    // host calls: rho and psi staged as the (-1:ni)^3 region of every block
    // ((ni+2)^3 values), on the device and in host buffers (pinned when the
    // driver grants it)
    double *d_rho = nullptr, *d_psi = nullptr;
    double *h_rho = nullptr, *h_psi = nullptr;
    bool h_pinned = false;
    double *d_gc = nullptr, *h_gc = nullptr;     // g interiors, device and pinned host staging
    cudaStream_t cs = nullptr;                   // the host call's copies and solve
    static constexpr int kGChunks = 8;           // arrays move in chunks, each gathered or scattered
    cudaEvent_t gev[kGChunks] = {};              // while the others are in flight
    cudaEvent_t pev[kGChunks] = {};
    std::string err;
};

static int check_device(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return SFM_EDEVICE;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return SFM_EDEVICE;
    if (prop.major != 10) return SFM_EDEVICE;   // built for sm_100a only
    return SFM_OK;
}

// Makes `dev` current for the lifetime of the guard and gives the caller's
// current device back on every return path: a host program that drives
// other GPUs finds its current device unchanged after a call.
struct DeviceGuard {
    int saved = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&saved) != cudaSuccess) {
            cudaGetLastError();
            saved = -1;
        }
        if (saved != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int now = -1;
        if (saved >= 0 && cudaGetDevice(&now) == cudaSuccess && now != saved) cudaSetDevice(saved);
    }
};

// true when p is device memory of device `dev` or managed memory: a host
// pointer or another GPU's memory handed to a kernel on `dev` would fault
// (or, where the GPU can reach host memory, silently use the wrong data)
static bool device_pointer_on(const void *p, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

extern "C" {

void sfm_default_params(sfm_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->bc = SFM_BC_PERIODIC;
    p->lmax = 3;
    p->precision = SFM_PREC_FP64;
    p->max_outer = 10;
    p->rel_tol = 1e-3;
    p->four_pi_G = 4.0 * 3.141592653589793;
    p->zero_mean = 1;
    p->ngh_io = 2;
    p->report_residual = 1;
    p->stagnation_exit = 1;
    p->profile = 0;
    p->rho_mask = 0.0;
    p->r_cloud = 0.0;
}

// No C++ exception may cross the C ABI: every entry point below runs its
// body under sfm_guard, which turns an exception into an error code
// (SFM_ENOMEM for a failed host allocation).
extern "C++" {
template <class F>
static int sfm_guard(F &&body) {
    try {
        return body();
    } catch (const std::bad_alloc &) {
        return SFM_ENOMEM;
    } catch (...) {
        return SFM_ECUDA;
    }
}
}

static int create_impl(const sfm_hier_desc *h, const sfm_params *p, sfm_ctx **out) {
    if (!h || !p || !out) return SFM_EINVAL;
    *out = nullptr;
    if (p->ngh_io < 1 || p->max_outer < 0 || p->max_outer > 1000 || !(p->rel_tol >= 0) ||
        p->bc < SFM_BC_PERIODIC || p->bc > SFM_BC_SPHERE_MHD_BE || !std::isfinite(p->rho_mask) ||
        !std::isfinite(p->r_cloud) ||
        (p->lmax != 3 && p->lmax != 4) ||
        (p->precision != SFM_PREC_FP64 && p->precision != SFM_PREC_MIXED))
        return SFM_EINVAL;
    {   // the hierarchy is validated on the host before any device work
        sfm::HostHier hh;
        int vr = hh.build(h);
        if (vr) return vr;
    }
    int rc = check_device();
    if (rc) return rc;
    std::unique_ptr<sfm_ctx> c(new sfm_ctx());
    c->p = *p;
    cudaGetDevice(&c->device);
    std::unique_ptr<sfm::SolverBase> s;
    if (p->precision == SFM_PREC_FP64) {
        auto *sd = new sfm::Solver<double>();
        s.reset(sd);
        rc = sd->init(h, p);
    } else {
        auto *sf = new sfm::Solver<float>();
        s.reset(sf);
        rc = sf->init(h, p);
    }
    if (rc) return rc;
    c->s = s.release();
    c->nb = h->nblocks; c->ni = h->ni; c->ngh = p->ngh_io;
    *out = c.release();
    return SFM_OK;
}

int sfm_create(const sfm_hier_desc *h, const sfm_params *p, sfm_ctx **out) {
    return sfm_guard([&] { return create_impl(h, p, out); });
}

// values of the (-1:ni)^3 region of every block: what the host-array entry
// point moves for rho and psi
static int64_t stage_elems(const sfm_ctx *c) {
    int64_t G = c->ni + 2;
    return (int64_t)c->nb * G * G * G;
}

int sfm_solve_device(sfm_ctx *c, const double *d_rho, double *d_psi, double *d_g, sfm_stats *st, void *stream) {
    if (!c || !c->s || !d_rho) return SFM_EINVAL;
    DeviceGuard dg(c->device);
    if (stream) {   // the stopping rule reads the residual on the host: no stream capture
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing((cudaStream_t)stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
            return SFM_EINVAL;
    }
    if (!device_pointer_on(d_rho, c->device) || (d_psi && !device_pointer_on(d_psi, c->device)) ||
        (d_g && !device_pointer_on(d_g, c->device)))
        return SFM_EINVAL;
    return sfm_guard([&] { return c->s->solve(d_rho, d_psi, d_g, st, (cudaStream_t)stream, 0, nullptr); });
}

}  // extern "C"

// fn(r0, r1) over rows [0, rows) on up to 16 host threads (at least 2^16
// rows each), an OpenMP team that stays alive between calls
template <class F>
static void host_rows(int64_t rows, const F &fn) {
    const int64_t per = (int64_t)1 << 16;
    const int nt = (int)std::max<int64_t>(1, std::min<int64_t>({16, (int64_t)omp_get_num_procs(), rows / per}));
#pragma omp parallel num_threads(nt)
    {
        const int t = omp_get_thread_num(), n = omp_get_num_threads();
        fn(rows * t / n, rows * (t + 1) / n);
    }
}
// a row of L doubles; a compile-time length makes the copy a few vector
// moves instead of a library call per row
template <int L>
static inline void copy_row_n(double *d, const double *s) {
    std::memcpy(d, s, L * sizeof(double));
}
// a row into the staging buffer: the staging rows are written once and
// then read by the copy engine only, so on x86-64 they go out as
// non-temporal 16-byte stores (no read of the destination lines into the
// cache before they are overwritten); d is 16-byte aligned (the staging
// buffer is, and every row holds an even number of values)
static inline void stream_row(double *d, const double *s, int len) {
#if defined(__x86_64__)
    if ((len & 1) == 0 && ((uintptr_t)d & 15) == 0) {
        for (int q = 0; q < len; q += 2) _mm_stream_pd(d + q, _mm_loadu_pd(s + q));
        return;
    }
#endif
    std::memcpy(d, s, (size_t)len * sizeof(double));
}
static inline void copy_row(double *d, const double *s, int len) {
    switch (len) {
        case 4: copy_row_n<4>(d, s); break;
        case 6: copy_row_n<6>(d, s); break;
        case 8: copy_row_n<8>(d, s); break;
        case 10: copy_row_n<10>(d, s); break;
        case 16: copy_row_n<16>(d, s); break;
        case 18: copy_row_n<18>(d, s); break;
        case 32: copy_row_n<32>(d, s); break;
        case 34: copy_row_n<34>(d, s); break;
        default: std::memcpy(d, s, (size_t)len * sizeof(double)); break;
    }
}

extern "C" {

// rows [row0, row1) of the g interiors [nblocks][3][ni^3] (a row = ni
// values) into the caller's [nblocks][3][(ni+2g)^3]; the io ghost layers of
// the caller's array are not touched
static void scatter_g_interiors(const double *src, double *g, int64_t row0, int64_t row1, int n, int gw) {
    const int Gi = n + 2 * gw;
    const int64_t Vi = (int64_t)Gi * Gi * Gi;
    host_rows(row1 - row0, [=](int64_t r0, int64_t r1) {
        for (int64_t r = row0 + r0; r < row0 + r1; r++) {
            const int64_t bc = r / ((int64_t)n * n);
            const int kj = (int)(r - bc * n * n), k = kj / n, j = kj - k * n;
            copy_row(g + bc * Vi + ((int64_t)(k + gw) * Gi + (j + gw)) * Gi + gw, src + r * n, n);
        }
    });
}

// rows [row0, row1) of the (-1:ni)^3 regions [nblocks][(ni+2)^3] (a row =
// ni+2 values) between the staging buffer and the caller's
// [nblocks][(ni+2g)^3]: gather (to_stage) or scatter; the caller's outer
// ghost layers (g >= 2) are never touched
static void stage_rows(double *stage, double *io, int64_t row0, int64_t row1, int n, int gw, bool to_stage) {
    const int Gc = n + 2, Gi = n + 2 * gw;
    const int64_t Vi = (int64_t)Gi * Gi * Gi;
    host_rows(row1 - row0, [=](int64_t r0, int64_t r1) {
        for (int64_t r = row0 + r0; r < row0 + r1; r++) {
            const int64_t b = r / ((int64_t)Gc * Gc);
            const int kj = (int)(r - b * Gc * Gc), k = kj / Gc, j = kj - k * Gc;
            double *o = io + b * Vi + ((int64_t)(k + gw - 1) * Gi + (j + gw - 1)) * Gi + (gw - 1);
            if (to_stage) stream_row(stage + r * Gc, o, Gc);
            else copy_row(o, stage + r * Gc, Gc);
        }
#if defined(__x86_64__)
        if (to_stage) _mm_sfence();   // the streamed rows are visible before the copy is queued
#endif
    });
}

static int stage_alloc(sfm_ctx *c, bool with_g) {
    const size_t bytes = (size_t)stage_elems(c) * sizeof(double);
    if (!c->d_rho) {
        if (cudaMalloc(&c->d_rho, bytes) != cudaSuccess || cudaMalloc(&c->d_psi, bytes) != cudaSuccess)
            return SFM_ENOMEM;
        c->h_pinned = cudaMallocHost(&c->h_rho, bytes) == cudaSuccess &&
                      cudaMallocHost(&c->h_psi, bytes) == cudaSuccess;
        if (!c->h_pinned) {   // ordinary host memory: the copies still work, without overlap
            cudaGetLastError();
            if (c->h_rho) cudaFreeHost(c->h_rho);
            c->h_rho = static_cast<double *>(std::malloc(bytes));
            c->h_psi = static_cast<double *>(std::malloc(bytes));
            if (!c->h_rho || !c->h_psi) return SFM_ENOMEM;
        }
    }
    if (!c->cs) {
        if (cudaStreamCreateWithFlags(&c->cs, cudaStreamNonBlocking) != cudaSuccess) return SFM_ECUDA;
        for (auto *ev : {c->gev, c->pev})
            for (int q = 0; q < sfm_ctx::kGChunks; q++)
                if (cudaEventCreateWithFlags(&ev[q], cudaEventDisableTiming) != cudaSuccess) return SFM_ECUDA;
    }
    if (with_g && !c->d_gc) {
        const size_t gbytes = (size_t)c->nb * 3 * c->ni * c->ni * c->ni * sizeof(double);
        if (cudaMalloc(&c->d_gc, gbytes) != cudaSuccess) return SFM_ENOMEM;
        if (cudaMallocHost(&c->h_gc, gbytes) != cudaSuccess) {
            c->h_gc = nullptr;
            return SFM_ENOMEM;
        }
    }
    return SFM_OK;
}

// The host-array call moves only what the solve uses: the (-1:ni)^3 region
// of rho and psi in ((ni+2)^3 of the (ni+2g)^3 values per block), that
// region of psi out, and g's interiors out.  Each array goes in chunks: the
// host threads gather chunk q+1 while chunk q is on the link, and scatter
// an output chunk as soon as it has landed.  Copies and solve are ordered
// on the context's copy stream.
static int solve_impl(sfm_ctx *c, const double *rho, double *psi, double *g, sfm_stats *st) {
    if (!c || !c->s || !rho) return SFM_EINVAL;
    DeviceGuard dg(c->device);
    int rc = stage_alloc(c, g != nullptr);
    if (rc) return rc;
    const int Gc = c->ni + 2, K = sfm_ctx::kGChunks;
    const int64_t rows = (int64_t)c->nb * Gc * Gc;
    auto chunk = [&](int64_t total, int q, int64_t &r0, int64_t &r1) {
        r0 = total * q / K;
        r1 = total * (q + 1) / K;
    };
    for (int q = 0; q < K; q++) {
        int64_t r0, r1;
        chunk(rows, q, r0, r1);
        const size_t off = (size_t)r0 * Gc, len = (size_t)(r1 - r0) * Gc * sizeof(double);
        stage_rows(c->h_rho, const_cast<double *>(rho), r0, r1, c->ni, c->ngh, true);
        if (cudaMemcpyAsync(c->d_rho + off, c->h_rho + off, len, cudaMemcpyHostToDevice, c->cs) != cudaSuccess)
            return SFM_ECUDA;
        if (psi) {
            stage_rows(c->h_psi, psi, r0, r1, c->ni, c->ngh, true);
            if (cudaMemcpyAsync(c->d_psi + off, c->h_psi + off, len, cudaMemcpyHostToDevice, c->cs) != cudaSuccess)
                return SFM_ECUDA;
        }
    }
    // g: the solve writes block interiors only, staged compact on the device
    // and scattered into the caller's array on the host -- its io ghost
    // layers keep the caller's values without a copy in
    c->s->gCompact = true;
    c->s->ioGw = 1;
    rc = c->s->solve(c->d_rho, psi ? c->d_psi : nullptr, g ? c->d_gc : nullptr, st, c->cs, 0, nullptr);
    c->s->gCompact = false;
    c->s->ioGw = 0;
    if (rc != SFM_OK && rc != SFM_ENOTCONVERGED) return rc;
    const int64_t grows = (int64_t)c->nb * 3 * c->ni * c->ni;
    // every output chunk is queued before the first is scattered
    for (int q = 0; q < K && psi; q++) {
        int64_t r0, r1;
        chunk(rows, q, r0, r1);
        const size_t off = (size_t)r0 * Gc, len = (size_t)(r1 - r0) * Gc * sizeof(double);
        if (cudaMemcpyAsync(c->h_psi + off, c->d_psi + off, len, cudaMemcpyDeviceToHost, c->cs) != cudaSuccess ||
            cudaEventRecord(c->pev[q], c->cs) != cudaSuccess)
            return SFM_ECUDA;
    }
    for (int q = 0; q < K && g; q++) {
        int64_t r0, r1;
        chunk(grows, q, r0, r1);
        if (cudaMemcpyAsync(c->h_gc + r0 * c->ni, c->d_gc + r0 * c->ni, (size_t)(r1 - r0) * c->ni * sizeof(double),
                            cudaMemcpyDeviceToHost, c->cs) != cudaSuccess ||
            cudaEventRecord(c->gev[q], c->cs) != cudaSuccess)
            return SFM_ECUDA;
    }
    for (int q = 0; q < K && psi; q++) {
        int64_t r0, r1;
        chunk(rows, q, r0, r1);
        if (cudaEventSynchronize(c->pev[q]) != cudaSuccess) return SFM_ECUDA;
        stage_rows(c->h_psi, psi, r0, r1, c->ni, c->ngh, false);
    }
    for (int q = 0; q < K && g; q++) {
        int64_t r0, r1;
        chunk(grows, q, r0, r1);
        if (cudaEventSynchronize(c->gev[q]) != cudaSuccess) return SFM_ECUDA;
        scatter_g_interiors(c->h_gc, g, r0, r1, c->ni, c->ngh);
    }
    if (st) {
        const int64_t sb = stage_elems(c) * (int64_t)sizeof(double);
        st->h2d_bytes = sb * (psi ? 2 : 1);
        st->d2h_bytes = (psi ? sb : 0) + (g ? grows * c->ni * (int64_t)sizeof(double) : 0);
    }
    return rc;
}

int sfm_solve(sfm_ctx *c, const double *rho, double *psi, double *g, sfm_stats *st) {
    return sfm_guard([&] { return solve_impl(c, rho, psi, g, st); });
}

int sfm_adjoint(sfm_ctx *c, const double *dJ_dphi, double *dJ_drho, sfm_stats *st) {
    if (!c || !c->s || !dJ_dphi || !dJ_drho) return SFM_EINVAL;
    DeviceGuard dg(c->device);
    return sfm_guard([&] { return c->s->adjoint(dJ_dphi, dJ_drho, st, nullptr); });
}

void sfm_destroy(sfm_ctx *c) {
    if (!c) return;
    DeviceGuard dg(c->device);
    if (c->d_rho) cudaFree(c->d_rho);
    if (c->d_psi) cudaFree(c->d_psi);
    if (c->h_pinned) {
        cudaFreeHost(c->h_rho);
        cudaFreeHost(c->h_psi);
    } else {
        std::free(c->h_rho);
        std::free(c->h_psi);
    }
    if (c->d_gc) cudaFree(c->d_gc);
    if (c->h_gc) cudaFreeHost(c->h_gc);
    for (auto *ev : {c->gev, c->pev})
        for (int q = 0; q < sfm_ctx::kGChunks; q++)
            if (ev[q]) cudaEventDestroy(ev[q]);
    if (c->cs) cudaStreamDestroy(c->cs);
    delete c->s;
    delete c;
}

const char *sfm_strerror(int code) {
    switch (code) {
        case SFM_OK: return "ok";
        case SFM_EINVAL: return "invalid argument";
        case SFM_EHIER: return "hierarchy violates a link-list invariant";
        case SFM_ECUDA: return "CUDA runtime error";
        case SFM_ENOMEM: return "out of memory";
        case SFM_ENOTCONVERGED: return "outer iteration did not reach rel_tol";
        case SFM_ENONFINITE: return "non-finite input";
        case SFM_EDEVICE: return "no usable sm_100 CUDA device";
        case SFM_ETIMEOUT: return "bounded device wait expired";
        case SFM_ESIZE: return "size exceeds a fixed maximum";
        default: return "unknown error";
    }
}

int sfm_autotune(sfm_ctx *c, int32_t reps, const double *d_rho) {
    if (!c || !c->s || reps < 1 || reps > 100) return SFM_EINVAL;
    DeviceGuard dg(c->device);
    if (d_rho && !device_pointer_on(d_rho, c->device)) return SFM_EINVAL;
    return sfm_guard([&] { return c->s->autotune(reps, d_rho); });
}

int sfm_tune_save(const sfm_ctx *c, char *buf, size_t cap, size_t *len) {
    if (!c || !c->s) return SFM_EINVAL;
    return sfm_guard([&] {
        const std::string t = c->s->tune_text();
        if (len) *len = t.size();
        if (!buf) return SFM_OK;
        if (cap < t.size() + 1) return SFM_ESIZE;
        std::memcpy(buf, t.c_str(), t.size() + 1);
        return SFM_OK;
    });
}

int sfm_tune_load(sfm_ctx *c, const char *text) {
    if (!c || !c->s || !text) return SFM_EINVAL;
    DeviceGuard dg(c->device);
    return sfm_guard([&] { return c->s->tune_load(text) ? SFM_OK : SFM_EINVAL; });
}

// Test hook (not part of include/sfmg.h; host code only, no device): parses
// a tuning table and writes it back in canonical form.  Returns the number
// of entries, SFM_EINVAL for a malformed table or SFM_ESIZE when `out` is
// too small.
int sfm_tune_text_check(const char *in, char *out, size_t cap) {
    return sfm_guard([&] {
        sfm::TuneTable t;
        if (!in || !t.parse(in)) return SFM_EINVAL;
        const std::string s = t.text();
        if (out) {
            if (cap < s.size() + 1) return SFM_ESIZE;
            std::memcpy(out, s.c_str(), s.size() + 1);
        }
        return (int)t.v.size();
    });
}

int sfm_info(const sfm_ctx *c, int32_t *fmg_levels, int64_t *device_bytes) {
    if (!c || !c->s) return SFM_EINVAL;
    if (fmg_levels) *fmg_levels = c->s->fmg_levels();
    if (device_bytes) *device_bytes = c->s->device_bytes();
    return SFM_OK;
}

// Test hook (not part of include/sfmg.h): poll limit of the smoother's
// consumer stage waits (k_relax_bulk); 0 makes every such wait give up at
// once, so a solve exercises the bounded-wait error path (SFM_ETIMEOUT).
int sfm_debug_set_wait_polls(sfm_ctx *c, uint32_t polls) {
    if (!c || !c->s) return SFM_EINVAL;
    c->s->set_wait_polls(polls);
    return SFM_OK;
}

// Test hooks (not part of include/sfmg.h): guard bands of `bytes` (rounded
// up to 4 KiB; 0 turns the mode off) around every device array of the
// contexts created from now on, in this process; and the number of band
// bytes a context's kernels have changed (-1 if they could not be read).
int sfm_debug_set_guard_bytes(uint64_t bytes) {
    if (bytes > ((uint64_t)1 << 30)) return SFM_EINVAL;
    sfm::g_guard_bytes.store((bytes + 4095) / 4096 * 4096);
    return SFM_OK;
}
int sfm_debug_check_guards(sfm_ctx *c, int64_t *bad_bytes) {
    if (!c || !c->s || !bad_bytes) return SFM_EINVAL;
    DeviceGuard dg(c->device);
    if (cudaDeviceSynchronize() != cudaSuccess) return SFM_ECUDA;
    *bad_bytes = c->s->guard_violations();
    return *bad_bytes < 0 ? SFM_ECUDA : SFM_OK;
}

// Test hook (not part of include/sfmg.h): 1 runs every red-black colour
// sweep one thread per block, the block's cells in the order of a serial
// sweep; a result bit-identical to the parallel kernels shows that no cell
// of a colour depends on another cell of the same colour (race check).
int sfm_debug_set_serial_relax(sfm_ctx *c, int on) {
    if (!c || !c->s) return SFM_EINVAL;
    c->s->set_serial_relax(on != 0);
    return SFM_OK;
}

// Test hook (not part of include/sfmg.h): 0 fills every level's ghost
// cells by the three directional passes, 1 (the default) by one launch per
// level where that is exact.  Both give bit-identical fields.
int sfm_debug_set_ghost_merge(sfm_ctx *c, int on) {
    if (!c || !c->s) return SFM_EINVAL;
    c->s->set_ghost_merge(on != 0);
    return SFM_OK;
}

// Test hook (not part of include/sfmg.h): like sfm_solve on host arrays, but
// stops after stage `stop_stage` (1 set-up, 2 first outer residual, 3 first
// fmg_lin, 4 outer loop) and copies that stage's level-0 field, ghost width 1,
// into `dump`.
int sfm_debug_solve(sfm_ctx *c, const double *rho, double *psi, double *g, sfm_stats *st, int stop_stage,
                    double *dump) {
    if (!c || !c->s || !rho) return SFM_EINVAL;
    if (stop_stage == 0) return sfm_solve(c, rho, psi, g, st);
    DeviceGuard dg(c->device);
    int rc = stage_alloc(c, false);
    if (rc) return rc;
    const int64_t rows = (int64_t)c->nb * (c->ni + 2) * (c->ni + 2);
    const size_t bytes = (size_t)stage_elems(c) * sizeof(double);
    stage_rows(c->h_rho, const_cast<double *>(rho), 0, rows, c->ni, c->ngh, true);
    if (cudaMemcpy(c->d_rho, c->h_rho, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return SFM_ECUDA;
    if (psi) {
        stage_rows(c->h_psi, psi, 0, rows, c->ni, c->ngh, true);
        if (cudaMemcpy(c->d_psi, c->h_psi, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return SFM_ECUDA;
    }
    (void)g;   // an early stop writes no g
    return sfm_guard([&] {
        c->s->ioGw = 1;
        const int r = c->s->solve(c->d_rho, psi ? c->d_psi : nullptr, nullptr, st, nullptr, stop_stage, dump);
        c->s->ioGw = 0;
        return r;
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// sfm_uniform_solve_noalloc: device address of the fixed scratch array,
// looked up once per device with that device current
// ---------------------------------------------------------------------------
namespace {
constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;
double *g_noalloc_ptr[kNoallocMaxDevices] = {};

int noalloc_scratch(int dev, double **out) {
    if (dev < 0 || dev >= kNoallocMaxDevices) return SFM_EDEVICE;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, sfm::g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return SFM_ECUDA;
        }
        g_noalloc_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return SFM_OK;
}

}  // namespace

extern "C" int sfm_uniform_solve_noalloc(const double *d_rho, double *d_psi, int n, double h, double four_pi_G,
                                         double rel_tol, int max_cycles, int *cycles, double *rel_residual,
                                         void *stream) {
    if (!d_rho || !d_psi) return SFM_EINVAL;
    if (n < 2 || n > sfm::NOALLOC_MAX_N || (n & (n - 1)) != 0) return SFM_ESIZE;
    if (!(h > 0.0) || !std::isfinite(h) || !std::isfinite(four_pi_G) || !(rel_tol >= 0.0) || max_cycles < 0 ||
        max_cycles > 1000)
        return SFM_EINVAL;
    if ((reinterpret_cast<uintptr_t>(d_rho) | reinterpret_cast<uintptr_t>(d_psi)) % alignof(double) != 0)
        return SFM_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cycles || rel_residual) {
        // the host outputs need a copy and a wait, which a stream under capture
        // forbids: refuse before any other runtime call (the capture stays valid)
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
            cudaGetLastError();
            return SFM_EINVAL;
        }
        if (cs != cudaStreamCaptureStatusNone) return SFM_EINVAL;
    }
    int rc = check_device();
    if (rc != SFM_OK) return rc;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return SFM_EDEVICE;
    if (!device_pointer_on(d_rho, dev) || !device_pointer_on(d_psi, dev)) return SFM_EINVAL;
    double *s = nullptr;
    rc = noalloc_scratch(dev, &s);
    if (rc != SFM_OK) return rc;
    const sfm::MgData d = sfm::noalloc_layout(s, n, h);
    double *out = s + sfm::noalloc_level_doubles(sfm::NOALLOC_MAX_N);
    sfm::k_mg_uniform_noalloc<<<1, 1024, 0, st>>>(d, d_rho, d_psi, four_pi_G, rel_tol, max_cycles, out,
                                                  (int64_t)sfm::noalloc_level_doubles(n));
    if (cudaGetLastError() != cudaSuccess) return SFM_ECUDA;
    if (!cycles && !rel_residual) return SFM_OK;
    double hv[2] = {0.0, 0.0};
    if (cudaMemcpyAsync(hv, out, sizeof hv, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return SFM_ECUDA;
    }
    if (cycles) *cycles = (int)hv[1];
    if (rel_residual) *rel_residual = hv[0];
    if (hv[1] < 0.0) return SFM_ENONFINITE;   // the kernel found a non-finite density
    return hv[0] <= rel_tol ? SFM_OK : SFM_ENOTCONVERGED;
}
