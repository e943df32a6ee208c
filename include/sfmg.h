/*
 * sfmg.h -- C ABI of the B200 self-gravity FMG Poisson solver.
 *
 * The solver is a drop-in for the reference's `fmg_poisson` entry point
 * (fmg.F90:63-74, public in module `fmg`, fmg.F90:23), which takes no
 * arguments and reads the block hierarchy from module globals of `grid`
 * (BlockMem(gid)%u, GidList, ParentGid/ChildGid/NeighborGid, CellWidth,
 * touch_boundary; grid.F90:19-66, boundary_fixed.F90:217-231).  The
 * replacement receives the same information explicitly: a hierarchy
 * descriptor (the link tables of grid.F90:44-52 in fmg-local numbering) and
 * per-block arrays laid out like BlockMem(gid)%u(:,:,:,m) (Fortran order,
 * i fastest, `ngh_io` ghost layers).  A Fortran host keeps the name
 * `fmg_poisson` through an ISO_C_BINDING shim that gathers these arrays and
 * calls sfm_solve.
 *
 * Conventions shared by every entry point:
 *   - blocks are numbered 0..nblocks-1 and must be sorted by AMR level
 *     (the reference's GidList(n, level), grid.F90:64);
 *   - face index  f = lr + 2*dir, lr 0 = Left, 1 = Right, dir 0/1/2 = x/y/z
 *     (NeighborGid(lr, dir), grid.F90:47);
 *   - child index c = lri + 2*lrj + 4*lrk (ChildGid(lri,lrj,lrk), grid.F90:50);
 *   - a block array holds (ni+2*ngh_io)^3 doubles, i fastest, so cell
 *     (i,j,k), -ngh_io <= i,j,k < ni+ngh_io, sits at
 *     ((k+ngh_io)*(ni+2*ngh_io) + (j+ngh_io))*(ni+2*ngh_io) + (i+ngh_io);
 *   - every function returns SFM_OK (0) or a negative SFM_E* code and never
 *     aborts the process (the reference prints and stops, fmg_data.F90:185,575).
 *
 * Threading: a context is used by one host thread at a time and owns all of
 * its device memory; it lives on the CUDA device that was current when it
 * was created.  Every call that takes a context makes that device current
 * for its duration and gives the caller's current device back before it
 * returns.
 */
#ifndef SFMG_H
#define SFMG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define SFM_OK               0
#define SFM_EINVAL          -1   /* bad argument (NULL pointer, bad size)      */
#define SFM_EHIER           -2   /* hierarchy violates a link-list invariant   */
#define SFM_ECUDA           -3   /* CUDA runtime error                         */
#define SFM_ENOMEM          -4   /* device or host allocation failed           */
#define SFM_ENOTCONVERGED   -5   /* outer loop ended without reaching rel_tol  */
#define SFM_ENONFINITE      -6   /* non-finite density or potential on input   */
#define SFM_EDEVICE         -7   /* no usable CUDA device / wrong architecture */
#define SFM_ETIMEOUT        -8   /* a bounded device wait gave up              */
#define SFM_ESIZE           -9   /* a size exceeds a fixed maximum             */

/* ---- hierarchy ---------------------------------------------------------
 * Replaces the link tables that fmg_make_linklist (fmg_data_if.F90:298-411)
 * gathers from module `grid`.  Parent-level neighbour links
 * (NeighborParentLevel, fmg_data_if.F90:376-395) are derived internally. */
typedef struct sfm_hier_desc {
    int32_t nlev;            /* AMR levels present: 0 .. nlev-1 (Lmin .. LevelMax) */
    int32_t nblocks;
    int32_t ni, nj, nk;      /* cells per block edge (NI,NJ,NK, config.h:15-17);
                                must be equal and a power of two >= 4            */
    int32_t ngb[3];          /* base blocks per dimension (NGI_BASE.., config.h:21-23) */
    const int32_t *level;    /* [nblocks] AMR level of each block                */
    const int32_t *ijk;      /* [3*nblocks] block index on its level (Igrid..)   */
    const int32_t *parent;   /* [nblocks] parent block, -1 on level 0            */
    const int32_t *child;    /* [8*nblocks] children, -1 for a block without any */
    const int32_t *nbr;      /* [6*nblocks] same-level face neighbour or -1      */
    const int8_t  *touch;    /* [6*nblocks] 1 where the face is on the physical
                                boundary (touch_boundary, boundary_fixed.F90:217) */
    const double  *cellwidth;/* [nlev] cell width h at fmg level 0 (CellWidth)   */
    const double  *x0;       /* [3*nblocks] coordinates of the centre of cell
                                (0,0,0) of each block (BlockMem(gid)%x(Imin)..)  */
} sfm_hier_desc;

/* ---- solver parameters ------------------------------------------------
 * The reference hard-codes these (fmg.F90:146,179; config.h:194). */
#define SFM_BC_PERIODIC 0   /* fmg_boundary_phys_periodic.F90                  */
#define SFM_BC_SPHERE   1   /* fmg_boundary_phys_sphere.F90 (multipole ghosts)  */
#define SFM_BC_ZMIRROR  2   /* fmg_boundary_phys_zmirror.F90: multipole ghosts,
                               a mirror plane on the box's z-min face          */
#define SFM_BC_CYL_ZPERIODIC  3  /* fmg_boundary_phys_cyl_zperiodic.F90: periodic
                               in z, the 2D potential a00 ln(r) on the x and y
                               faces, the source masked outside a cylinder  */
#define SFM_BC_MASK_ZPERIODIC 4  /* fmg_boundary_phys_mask_zperiodic.F90: as 3,
                               the source masked below params.rho_mask      */
#define SFM_BC_SPHERE_MHD_BE  5  /* fmg_boundary_phys_sphere_MHD_BE.F90: as 1,
                               the source masked outside params.r_cloud     */
#define SFM_PREC_FP64   0   /* every operation in FP64, as the reference       */
#define SFM_PREC_MIXED  1   /* FP32 inner fmg_lin/vmg, FP64 outer loop and base solve */

typedef struct sfm_params {
    int32_t bc;              /* SFM_BC_*                                        */
    int32_t lmax;            /* multipole order for SFM_BC_SPHERE / _ZMIRROR: 3
                                (reference) or 4                                */
    int32_t precision;       /* SFM_PREC_*                                      */
    int32_t max_outer;       /* nfmgmax (reference: 10)                         */
    double  rel_tol;         /* errormax (reference: 1e-3)                      */
    double  four_pi_G;       /* MP_Gconst * Pi4 (fmg_data_if.F90:40)            */
    int32_t zero_mean;       /* ZERO_AVERAGE_DENSITY (config.h:194): subtract the
                                leaf-volume mean of rho and zero the base mean  */
    int32_t ngh_io;          /* ghost layers of the caller's block arrays, >= 1
                                (N_GHOST_CELL = 2, config.h:135)                */
    int32_t report_residual; /* 1: compute the true FP64 composite residual of
                                the returned potential into sfm_stats          */
    int32_t stagnation_exit; /* 1: stop when the ratio fails to halve, as
                                fmg.F90:193 does; 0: run until rel_tol/max_outer */
    int32_t profile;         /* 1: time every smoother launch on fmg level 0
                                with CUDA events (sfm_stats.smoother_*)        */
    double  rho_mask;        /* SFM_BC_MASK_ZPERIODIC: the source (4 pi G rho)
                                is set to 0 where it is below this value
                                (MP_rhomask, fmg_boundary_phys_mask_zperiodic.F90:129) */
    double  r_cloud;         /* SFM_BC_SPHERE_MHD_BE: the source is set to 0 at
                                x^2+y^2+z^2 >= r_cloud^2 (Rcloud,
                                fmg_boundary_phys_sphere_MHD_BE.F90:72)       */
} sfm_params;

/* Fills *p with the reference's defaults (periodic, FP64, 10 outer
 * iterations, rel_tol 1e-3, 4piG = 4pi, zero_mean on, ngh_io 2). */
void sfm_default_params(sfm_params *p);

#define SFM_MAX_HISTORY 64
typedef struct sfm_stats {
    int32_t outer_iters;         /* fmg_lin calls done                        */
    int32_t converged;           /* bool_converge of fmg_cycle (fmg.F90:181)  */
    double  resh2max;            /* max_leaf |h^2 SRC| (fmg.F90:172)          */
    double  ratio[SFM_MAX_HISTORY]; /* Resh2maxg/resh2max per iteration (fmg.F90:188) */
    double  true_rel_residual;   /* max_leaf|h^2 (SRC - L phi)| / resh2max    */
    double  rho_mean;            /* subtracted mean of 4 pi G rho             */
    double  device_ms;           /* device time of the solve (CUDA events)   */
    int64_t kernel_launches;     /* kernels launched by this call             */
    double  smoother_ms;         /* summed duration of the level-0 red-black
                                    colour launches (params.profile = 1)      */
    int64_t smoother_launches;   /* number of those launches                  */
    int64_t smoother_cells;      /* leaf cells swept per launch x launches    */
    int32_t elem_bytes;          /* bytes per value of the inner solve (8 or 4) */
    int32_t smoother_colours;    /* red-black colours per timed launch: 1, or
                                    2 x the local sweeps when the mixed
                                    schedule fuses them                       */
    int64_t h2d_bytes;           /* sfm_solve: bytes copied host to device    */
    int64_t d2h_bytes;           /* sfm_solve: bytes copied device to host
                                    (0 for the device-array call)             */
} sfm_stats;

typedef struct sfm_ctx sfm_ctx;

/* Builds the device hierarchy, neighbour and work tables and allocates all
 * device fields (fmg_data_init + fmg_alloc_LoL + fmg_make_linklist,
 * fmg_data.F90:110-319, fmg_data_if.F90:298-411).  The link invariants of
 * fmg_check_linklist (fmg_data_if.F90:415-568) are verified; a violation
 * returns SFM_EHIER. */
int sfm_create(const sfm_hier_desc *h, const sfm_params *p, sfm_ctx **out);

/* One solve with HOST arrays: replaces fmg_poisson (fmg.F90:63-74).
 *   rho [nblocks][(ni+2g)^3]   density (U1(MRHO), fmg_data_if.F90:51), read on (-1:ni)^3
 *   psi [nblocks][(ni+2g)^3]   in: warm start U(MPSI) (fmg_data_if.F90:46), read on (-1:ni)^3
 *                              out: potential on (-1:ni)^3 (fmg_restore_u, fmg_data_if.F90:275-294)
 *   g   [nblocks][3][(ni+2g)^3] out: -grad phi on the interior (fmg_psi2g, fmg_poisson.F90:4-49);
 *                              entries outside the interiors are left as they are;
 *                              may be NULL
 *   st  may be NULL.
 * Returns SFM_OK, or SFM_ENOTCONVERGED when the outer loop stopped early
 * (the outputs are still written, as the reference continues in that case). */
int sfm_solve(sfm_ctx *c, const double *rho, double *psi, double *g, sfm_stats *st);

/* Same with DEVICE pointers on the context's device (no host copies).
 * `stream` is a cudaStream_t or NULL for the context's own stream.  Each
 * pointer must be device memory of the context's device (or managed
 * memory); a host pointer or another GPU's memory returns SFM_EINVAL.
 * The call waits for the stream between outer iterations (the stopping
 * rule reads the residual on the host), so it cannot be captured into a
 * caller's graph: a stream under capture returns SFM_EINVAL untouched. */
int sfm_solve_device(sfm_ctx *c, const double *d_rho, double *d_psi, double *d_g,
                     sfm_stats *st, void *stream);

/* Adjoint of the solve: given dJ/dphi on the interior of every block
 * (layout as psi; ghost entries ignored; entries on covered blocks act
 * through the restriction that defines phi there), returns dJ/drho on the
 * interior of every block (layout as rho) for the linear map rho -> phi that
 * sfm_solve converges to.  No counterpart in the reference.
 *   - The map is the fixed point of the solve's FP64 outer residual
 *     (fmg_poisson_resid at fmg level 0, fmg_poisson.F90:217-265, with the
 *     bilinear ghost fill and reflux); its transpose is applied exactly,
 *     operation by operation, and A^T lambda = dJ/dphi is solved by FGMRES
 *     preconditioned with this context's fmg_lin (FP32 inside when
 *     precision is SFM_PREC_MIXED).  The isolated-sphere boundary
 *     (multipoles of the masked source), the mask and the mean removal are
 *     chained back to rho.
 *   - params.rel_tol is the tolerance on ||dJ/dphi - A^T lambda||_2 relative
 *     to ||dJ/dphi||_2; params.max_outer caps the Krylov iterations.
 *   - dJ/drho is zero on covered blocks (the solve overwrites rho there by
 *     restriction) and on ghost entries.  With periodic boundaries phi's
 *     constant is free: dJ/dphi is taken orthogonal to constants.
 *   - The first call allocates the Krylov vectors (as many as fit, up to 30
 *     restarts' worth, in 80% of the free device memory).
 *   - Results are reproducible to roundoff, not bitwise (FP64 atomics).
 *   - Periodic and sphere boxes only: the other boundaries return SFM_EINVAL.
 * st: outer_iters = Krylov iterations, ratio[] = their residual history,
 * true_rel_residual = the final true relative residual. */
int sfm_adjoint(sfm_ctx *c, const double *dJ_dphi, double *dJ_drho, sfm_stats *st);

void sfm_destroy(sfm_ctx *c);
const char *sfm_strerror(int code);

/* Number of fmg sub-block levels (FMG_LevelMax+1, fmg_data.F90:113) and
 * bytes of device memory held by the context. */
int sfm_info(const sfm_ctx *c, int32_t *fmg_levels, int64_t *device_bytes);

/* ---- autotuner (no counterpart in the reference) -----------------------
 * Two kinds of knobs.
 *  - Launch shapes: ghost fill of a level by three directional passes or by
 *    one launch, threads of the smoother CTA, blocks per residual CTA.  Every
 *    variant evaluates the same expressions in the same order, so no choice
 *    changes a result bit.
 *  - The schedule of the mixed path's FP32 inner solve: V-cycles per level
 *    and sweeps of fmg_lin (the reference's fixed Ncycle = 2, Npre = Npost =
 *    2, fmg.F90:280-288), sweeps of vmg_fas (vmg.F90:125-135) and the cap on
 *    the base-grid defect corrections (mg.F90:50-52).  That solve only
 *    preconditions the FP64 defect correction, which converges to the same
 *    potential (within rel_tol) whatever the schedule; only its cost and the
 *    number of outer iterations change.  The FP64 path always runs the
 *    reference's schedule.
 *
 * sfm_autotune times every launch-shape candidate the context's hierarchy
 * uses (each `reps` times, 1 <= reps <= 100, on the context's own stream and
 * fields; the fields are zeroed first) and keeps the fastest.  With d_rho (a
 * density in sfm_solve_device's layout, device memory of the context's
 * device) a mixed-precision context also tunes the schedule by complete
 * solves of that density: from the reference's schedule, one knob at a
 * time, a change is kept only when the solve still converges to rel_tol and
 * is at least 2% faster (a few seconds for 1e5 blocks).  Call it between
 * solves, outside stream capture.  Without it (or after sfm_tune_load(c,
 * "")) the built-in launch shapes and the reference's schedule apply. */
int sfm_autotune(sfm_ctx *c, int32_t reps, const double *d_rho);

/* The tuning table as text, one choice per line
 *   "<knob> <element bytes> <block edge> <AMR level> <fill kind> <choice>",
 * '#' starting a comment line.  sfm_tune_save writes it NUL-terminated into
 * buf (when buf is not NULL) and its length without the NUL into *len (when
 * len is not NULL); SFM_ESIZE if cap is too small.  sfm_tune_load replaces
 * the table; a malformed table returns SFM_EINVAL and leaves it unchanged.
 * A table saved for one hierarchy and GPU may be loaded into a context of
 * another: unused entries are ignored, missing ones take the defaults. */
int sfm_tune_save(const sfm_ctx *c, char *buf, size_t cap, size_t *len);
int sfm_tune_load(sfm_ctx *c, const char *text);

/* Uniform periodic base-grid solve that allocates nothing.  No counterpart
 * in the reference: it runs the reference's base-grid multigrid (mg_cycle's
 * residual / mg_lin / correction loop, mg.F90:42-94, with mg_lin of
 * mg.F90:106-218) for callers that cannot allocate device memory when they
 * need a solve: code inside a fixed memory pool or a start-up arena, a
 * real-time step in which an allocator call would synchronise the device,
 * a host library that promises a fixed device footprint.
 *   d_rho, d_psi  device arrays of n^3 doubles, x fastest; psi is written
 *                 (it starts from zero: no warm start)
 *   n             cells per edge, a power of two, 2 <= n <= SFM_NOALLOC_MAX_N;
 *                 larger n returns SFM_ESIZE
 *   h, four_pi_G  cell width and the source factor: lap(psi) = four_pi_G (rho - mean rho)
 *   rel_tol, max_cycles  stop when max|residual| <= rel_tol * max|four_pi_G (rho - mean)|,
 *                 or after max_cycles mg_lin cycles (0 <= max_cycles <= 1000)
 *   cycles, rel_residual  host outputs, may be NULL; when either is given the
 *                 call waits for `stream` and returns SFM_ENOTCONVERGED if
 *                 rel_tol was not reached; when both are NULL it returns
 *                 after queueing the work.  A stream under capture cannot be
 *                 waited for: with either output given on such a stream the
 *                 call returns SFM_EINVAL without touching the stream, so
 *                 pass NULL for both there
 *   stream        a cudaStream_t, or NULL for the legacy default stream
 * A NaN or Inf anywhere in rho sets psi to NaN everywhere; with host
 * outputs the call then returns SFM_ENONFINITE (*cycles = -1).
 * d_rho and d_psi must be device memory of the current device (or managed
 * memory): anything else returns SFM_EINVAL.
 * Working arrays live in one fixed device array of the library (about
 * 2 MiB, enough for n = 32), cleared by the kernel itself before use, so
 * nothing needs zeroing and nothing carries over between calls.  There is
 * one such array per device: calls on one device whose executions overlap
 * (unordered streams, concurrent host threads) race and give wrong results.
 * The first call on each device looks up the array's address; make it
 * before any stream capture on that device.  Uses the current device. */
#define SFM_NOALLOC_MAX_N 32
int sfm_uniform_solve_noalloc(const double *d_rho, double *d_psi, int n, double h, double four_pi_G,
                              double rel_tol, int max_cycles, int *cycles, double *rel_residual,
                              void *stream);

/* Links of a block hierarchy computed on the device from the blocks' levels
 * and integer positions.  Replaces the link updates the reference runs after
 * each refinement (update_neighbor, update_neighbor_linklist,
 * update_parent_linklist; grid.F90:587-731), whose ParentGid / ChildGid /
 * NeighborGid fmg_make_linklist then reads (fmg_data_if.F90:298-411): the
 * arrays it fills are sfm_hier_desc's parent, child, nbr and touch, in the
 * same conventions, so a hierarchy regridded on the device is linked without
 * a round trip through the host.
 *   nblocks, nlev   blocks (any order) and AMR levels (nlev <= 16)
 *   d_level[nb]     AMR level of each block
 *   d_ijk[3*nb]     integer position of each block on its level, 0 <= i <
 *                   ngb[0] << level (likewise j, k; ngb[d] << (nlev-1) <= 2^20)
 *   ngb[3], periodic[3]  base blocks per direction and periodic flags (host)
 *   outputs d_parent[nb] (-1 on the base level), d_child[8*nb] (child
 *                   lri + 2 lrj + 4 lrk, -1 for a leaf), d_nbr[6*nb] (face
 *                   lr + 2 dir, the same-level neighbour, periodic directions
 *                   wrapping, else -1), d_touch[6*nb] (1 on the physical
 *                   boundary of a non-periodic direction)
 *   stream          a cudaStream_t, or NULL; the call waits for it, so a
 *                   stream under capture returns SFM_EINVAL
 * All arrays are device memory of the current device (else SFM_EINVAL).
 * Returns SFM_EHIER for a block outside its level's box, a block given
 * twice, a block above the base level without a parent, or a block with
 * some but not all of its 8 children. */
int sfm_link_blocks(int32_t nblocks, int32_t nlev, const int32_t *d_level, const int32_t *d_ijk,
                    const int32_t ngb[3], const int32_t periodic[3], int32_t *d_parent, int32_t *d_child,
                    int32_t *d_nbr, int8_t *d_touch, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* SFMG_H */
