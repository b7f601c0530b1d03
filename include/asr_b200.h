/* asr_b200.h -- C ABI of the B200 (sm_100a) augmented-space recursion library.
 *
 * A drop-in for the recursion hot path of mavensgroup/asr behind its site-class operator interface.  Every entry point
 * names the reference interface it replaces (paths relative to the asr project root).  Conventions:
 *   - every call returns an int status (ASR_OK = 0); asr_last_error() gives the message of the calling host thread;
 *   - arrays cross the ABI in Fortran (column-major) layout with the reference's shapes, so a Fortran caller passes its
 *     arrays through iso_c_binding unchanged; stored site / node / operation indices are 1-based as in the reference;
 *   - complex arrays are interleaved (re, im) doubles (Fortran complex(dp));
 *   - pointers are host pointers unless the name ends in _dev;
 *   - the caller owns every host buffer; device buffers belong to the context or the operator.
 * Errors are status codes, never aborts (the reference uses `error stop`).
 */
#ifndef ASR_B200_H
#define ASR_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ASR_OK 0
#define ASR_EINVAL 1    /* invalid argument (the reference's `error stop` on bad input) */
#define ASR_ENOMEM 2    /* device allocation failed */
#define ASR_ECUDA 3     /* CUDA runtime error */
#define ASR_ETIMEOUT 4  /* a bounded device wait gave up */
#define ASR_EEDGE 5     /* the closure reached the edge of the site cluster (src/asr_augcls.f90:672,676) */
#define ASR_ESTATE 6    /* an internal invariant failed (stabiliser size, hash table capacity) */

#define ASR_MODE_PLAIN 0 /* real Lanczos on H (src/reference/asr_recursion.f90:17-58): one chain per group */
#define ASR_MODE_EDC 1   /* complex-symmetric Lanczos on z - H(z) per energy (src/asr_edc.f90:75-164, :237-316) */

#define ASR_TAIL_NONE 0  /* cf_species tails, src/asr_chain.f90:18-23 */
#define ASR_TAIL_HULL 1
#define ASR_TAIL_BP 2
#define ASR_TAIL_AVG2 3

#define ASR_FP64 0       /* FP64 vectors and matvec */
#define ASR_FP32 1       /* FP32 vector storage and matvec, FP64 coefficients, reductions and fractions */

typedef struct asr_ctx asr_ctx;
typedef struct asr_op asr_op;

/* ---- library and context ---------------------------------------------------------------------------------------- */
int asr_version(void);
/* message of the last failed call on this host thread (src/asr_mpi.F90:191-197 par_fail replaced by status codes) */
int asr_last_error(char* buf, size_t n);
/* device context: stream, workspace.  One per host thread and device. */
int asr_ctx_create(int device, asr_ctx** ctx);
int asr_ctx_destroy(asr_ctx* ctx);
int asr_ctx_sync(asr_ctx* ctx);
/* chain statistics of the context (ed_nchain, ed_nlev, ed_nfall of src/asr_chain.f90:14-17) */
int asr_ctx_stats(const asr_ctx* ctx, int64_t* nchain, int64_t* nlev, int64_t* nfall);
/* run on the caller's CUDA stream (a cudaStream_t, e.g. the current stream of a PyTorch process); NULL: the context's own.
 * No counterpart in the reference (which has no device). */
int asr_ctx_set_stream(asr_ctx* ctx, void* stream);
/* per-launch CUDA-event timing of the hot kernels (the timer buckets of src/asr_runstats.f90:1-96 on the device):
 * on = 1 starts (and clears) it; asr_ctx_kernel_stats returns the summed device time, the launches and the algorithmic
 * bytes and flops of the chain step operator's launches, asr_ctx_kernel_stats_kind the same for one kernel kind */
enum {
  ASR_KERNEL_STEP = 0,      /* chain step operator (S application, diagonal terms, a-dot) */
  ASR_KERNEL_LANCZOS = 1,   /* Lanczos update w = y - a u - b u', projection, b-dot */
  ASR_KERNEL_KPM = 2,       /* KPM Chebyshev step (block matvec, recurrence, moments) */
  ASR_KERNEL_ADJOINT = 3,   /* one level of the adjoint's reverse sweep (all its kernels; the four kinds below split it) */
  ASR_KERNEL_ADJ_STEP = 4,  /* reverse sweep: the operator applied to wbar (fused step kernel with the ubar epilogue) */
  ASR_KERNEL_ADJ_VEC = 5,   /* reverse sweep: the vector updates (wbar = P(...), and ybar, ubar where not fused) */
  ASR_KERNEL_ADJ_GRAD = 6,  /* reverse sweep: the parameter gradient partials and their per-tile sums */
  ASR_KERNEL_ADJ_SCAL = 7,  /* reverse sweep: per-lane dot sums and the recurrence scalars */
  ASR_KERNEL_KINDS = 8
};
int asr_ctx_profile(asr_ctx* ctx, int on);
/* on = 1: the batched chain runs (asr_chains_run and its lane and device forms) and the adjoint (asr_chains_adjoint,
 * asr_chains_adjoint_ext) keep their device vector memory (one slab, at most half of the device memory free when it is
 * first needed, grown when a later call needs more) in the context after they return and reuse it on the next call,
 * instead of allocating and freeing it per call; on = 0 (the default) frees it.  For loops that run many chain sets or
 * gradients on one operator.  No counterpart in the reference (whose arrays are allocated per call). */
int asr_ctx_hold_workspace(asr_ctx* ctx, int on);
int asr_ctx_kernel_stats(asr_ctx* ctx, double* ms, int64_t* launches, double* bytes, double* flops);
int asr_ctx_kernel_stats_kind(asr_ctx* ctx, int kind, double* ms, int64_t* launches, double* bytes, double* flops);
/* number of kernels this context has launched (all kinds) */
int asr_ctx_launches(asr_ctx* ctx, int64_t* launches);

/* ---- operator: replaces augcls_op and build_augcls_operator (src/asr_augcls.f90:45-68, :596-823) ---------------- *
 * graph (graph_t, src/asr_augspace.f90:22-25): nbr_ptr(nsite+1), nbr(*) 1-based (0: no bond on the slot, -1: beyond the
 * cluster).  Model (class_alloy_t, :36-43): nsc(ncls), spc(ldspc, ncls), conc(ldspc, ncls), nsp species,
 * block(9, 9, nblock_slots, ntype_blocks), block0(9, 9, ntype_blocks) (NULL: zero).  cls(nsite), perm(nsite, nop),
 * dmat(9, 9, nop), start site, maxlevel, maxrank (0: unlimited), flippable(nsite) (NULL: all), stype(nsite) (NULL: 1).
 * The closure and every node table are built on the device; the node numbering equals the reference's serial order. */
int asr_op_build(asr_ctx* ctx, int nsite, const int* nbr_ptr, const int* nbr, int ncls, const int* nsc, const int* spc,
                 int ldspc, const double* conc, int nsp, const int* cls, const int* perm, int nop, const double* dmat,
                 int start, int maxlevel, int maxrank, const int* flippable, const int* stype, const double* block,
                 int nblock_slots, int ntype_blocks, const double* block0, asr_op** op);
/* build_augcls_operator with its optional targets (src/asr_augcls.f90:589-596, :808-820): for target graph site tsite(t)
 * and local state k = 0 .. nsc - 1 (the site alone in state k, every other site in its reference state),
 * tnode(k + 1, t) = the representative node (1-based; 0: not in the node set or the site cannot flip) and tgop(k + 1, t)
 * the operation that maps the node onto it (1-based), both (nsmax, ntarget) with nsmax = max(nsc). */
int asr_op_build_targets(asr_ctx* ctx, int nsite, const int* nbr_ptr, const int* nbr, int ncls, const int* nsc, const int* spc,
                         int ldspc, const double* conc, int nsp, const int* cls, const int* perm, int nop, const double* dmat,
                         int start, int maxlevel, int maxrank, const int* flippable, const int* stype, const double* block,
                         int nblock_slots, int ntype_blocks, const double* block0, const int* tsite, int ntarget, int* tnode,
                         int* tgop, asr_op** op);
/* augcls_free (src/asr_augcls.f90:569-585) */
int asr_op_free(asr_op* op);
/* dims: nn, nslot, nsmax, nop, ncls, ntype, nstab, nsp */
int asr_op_dims(const asr_op* op, int* dims);
/* host copies of the node tables in the reference layout: flipr/flipg(nsmax, nn), hopr/hopg(nslot, nn), lst, site,
 * ncl, level (nn), norb, sq (nn), stab_ptr(nn+1), stab(nstab).  Any pointer may be NULL. */
int asr_op_export_tables(const asr_op* op, int* flipr, int* flipg, int* hopr, int* hopg, int* lst, int* site, int* ncl,
                         int* level, double* norb, double* sq, int* stab_ptr, int* stab);

/* ---- per-operator state: augcls_set_params :121, augcls_freeze_site/_any :129/:147, augcls_set_start :107,
 *      augcls_set_chi :165, augcls_set_class_conc :178 --------------------------------------------------------------- */
int asr_op_set_params(asr_op* op, const double* c, const double* d, const double* o, const double* e);
/* augcls_freeze_site (src/asr_augcls.f90:129-142): every node on `site` takes the parameters of species sp (1..nsp);
 * when the site is the start site, sp must belong to the start node's class.  The nodes must sit on a site that was not
 * flippable when the node set was built.  The tables a freeze reads are copied to the host on the first freeze of the
 * operator; later freezes only upload the frozen array (on the context's stream, no synchronisation). */
int asr_op_freeze_site(asr_op* op, int site, int sp);
/* augcls_freeze_any (src/asr_augcls.f90:147-161): the same for any species index 1..nsp (a path species, the partner of a
 * pair); nfound (optional) receives the number of nodes on the site (0: the site lies outside the node set) */
int asr_op_freeze_any(asr_op* op, int site, int sp, int* nfound);
int asr_op_unfreeze(asr_op* op);
int asr_op_set_start(asr_op* op, int l0);
int asr_op_set_chi(asr_op* op, const double* chi);
int asr_op_set_class_conc(asr_op* op, int kap, const double* conc);

/* ---- application: the linop interface (src/asr_operator.f90:10-28) -------------------------------------------------- */
/* augcls_apply (src/asr_augcls.f90:275-297): y = H x for nvec real vectors x(9 nn, nvec), normalised coordinates */
int asr_op_apply(asr_op* op, const double* x, double* y, int nvec);
/* augcls_hp_c (src/asr_augcls.f90:301-320): y = h x = (c + D S D) x for nvec complex vectors x(9 nn, nvec) in normalised
 * coordinates with the operator's c and d (o and e not applied; the route ed3's h') */
int asr_op_hp_c(asr_op* op, const double* x, double* y, int nvec);
/* augcls_rand_c (:419-446): w = X x, complex parameters par(9, nsp), complex x(9 nn, nvec) */
int asr_op_rand_c(asr_op* op, const double* par, const double* x, double* w, int nvec);
/* augcls_project_c (:329-348), in place on complex x(9 nn, nvec) */
int asr_op_project_c(asr_op* op, double* x, int nvec);

/* ---- batched chains: chain_greens / edc_green_blk / lanczos (src/asr_class_scf.f90:966-1160, src/asr_edc.f90:237-316,
 *      src/reference/asr_recursion.f90:17-58) ------------------------------------------------------------------------ */
typedef struct {
  const double* c;   /* (9, nsp) operator parameters of the chain: H = E_nu + h - h o h, h = c + d S d, E_nu = e */
  const double* d;
  const double* o;
  const double* e;
  const double* pa;  /* (9, nsp) energy-dependent diagonal X(z) = z pa + pb (edc mode), NULL: zero */
  const double* pb;
  int frozen_sp;     /* species frozen on the start site (0: none), augcls_freeze_site(op, start, sp) */
  int start_orb;     /* start orbital l0 (1..9): start vector e_(node 1, l0), chi(g) = dmat(l0, l0, g) */
  int nlev;          /* chain depth (recursion steps) */
  int reserved;
} asr_chain_group;

/* Runs every chain of the batch: in ASR_MODE_EDC one chain per (group, energy), in ASR_MODE_PLAIN one real chain per
 * group whose terminated fraction is evaluated at every energy.  z(nz) complex energies; outputs g(nz, ngroup) complex;
 * optional a, b (nlevmax, nz, ngroup) complex (plain mode: (nlevmax, 1, ngroup)), mused (nz, ngroup).
 * depth_tol > 0: adaptive depth (src/asr_edc.f90:121-127).  tail: ASR_TAIL_*; in plain mode ASR_TAIL_BP is the real
 * Beer-Pettifor asymptote (src/reference/asr_terminator.f90:39-67) and ASR_TAIL_AVG2 'sqrt-avg2'.  project: project each
 * new Lanczos vector on the symmetric subspace (src/asr_chain.f90:24-26). */
int asr_chains_run(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const double* z, int nz, int mode,
                   double depth_tol, int tail, int precision, int project, double* g, double* a, double* b, int* mused);
/* Same, with z and g already in device memory (double2 arrays); a, b, mused host pointers or NULL. */
int asr_chains_run_dev(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const void* z_dev, int nz,
                       int mode, double depth_tol, int tail, int precision, int project, void* g_dev, double* a, double* b,
                       int* mused);

/* The tasks of chain_worker (src/asr_class_scf.f90:1071-1160) as explicit lanes of the edc route: lane L runs group
 * lane_group[L] (1-based) at the energy lane_z[L] (complex), so that a rank runs exactly its share of the cyclic task split
 * (:1095-1097; energy blocks of a group need not be contiguous or the same for every group).  g(nlane) complex,
 * mused(nlane) optional.  The _dev form takes device arrays of lane energies and results (lane_group stays on the host);
 * results are bitwise those of asr_chains_run for the same (group, energy). */
int asr_chains_run_lanes(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const int* lane_group,
                         const double* lane_z, int nlane, double depth_tol, int tail, int precision, int project, double* g,
                         int* mused);
int asr_chains_run_lanes_dev(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const int* lane_group,
                             const void* lane_z_dev, int nlane, double depth_tol, int tail, int precision, int project,
                             void* g_dev);

/* dos_final (src/asr_class_scf.f90:1912-1931): the l-resolved DOS on the real axis.  edos_e(ndos) = emin + (emax - emin)
 * (ie - 1) / max(ndos - 1, 1); the edc chains of every group at z = edos_e + i eta (as asr_chains_run); then
 * edos(ie, l, comp, spin) = sum over the groups q with comp(q), spin(q) (1-based) and lorb(q) = l (0 s, 1 p, 2 d) of
 * -worb(q) Im G_q / pi, worb the orbital-group sizes (lorbk, worbk of the reference).  edos (ndos, 3, ncomp, nspin). */
int asr_dos_final(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const int* comp, const int* spin,
                  const int* lorb, const double* worb, int ncomp, int nspin, double emin, double emax, double eta, int ndos,
                  double depth_tol, int tail, int precision, double* edos_e, double* edos);

/* edc_green_proj (src/asr_edc.f90:174-232) for every (group, energy): each chain runs its full depth (no depth test) and
 * every Lanczos vector is projected on the target states, cpr(k, l, t) = sum_ks tw(l, ks, t) psi_k(node ks of t, l) with
 * psi the unreduced amplitude (augcls_amp_c, src/asr_augcls.f90:251-261); gp(l, t) = sum_k cpr(k, l, t) pv_k with pv of
 * cf_species, gp4 the same with the chain cut four steps earlier.  tnode, tgop (nsmax, nt) as returned by
 * asr_op_build_targets; tw (9, nsmax, nt, ngroup) dressing weights per group (spectral_dressing, src/asr_spectral.f90:200-229).
 * Outputs g (nz, ngroup), gp and gp4 (9, nt, nz, ngroup) complex, mused (nz, ngroup) or NULL. */
int asr_chains_proj(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const double* z, int nz, int tail,
                    int precision, int project, int nt, const int* tnode, const int* tgop, const double* tw, double* g,
                    double* gp, double* gp4, int* mused);

/* epi_blocks (src/asr_epi.f90:639-663), the chains of the effective pair interactions, for every (group, energy): v9(9, ngroup)
 * the symmetry-adapted start vector of each group on the start node (epi_adapted, unit norm) and chi(nop, ngroup) its
 * characters under the operator's group (+-1).  Two full-depth chains of the edc route per (group, energy): from s0 with
 * the projection on |v> = h'|s0> (projected, h' = c + d S d), and from |v>/|v| with the projection on s0 (a chain that
 * closes gets no tail).  x(4, nz, ngroup) complex = X0 = <s0|G|s0>, X1 = <s0|h'G|s0> (the mean of the two chains),
 * X2 = <s0|h'Gh'|s0> and the X1 mismatch of the two chains; mused(2, nz, ngroup) the two depths, or NULL.  Operator-level
 * frozen sites (asr_op_freeze_site: the path site and the partner) apply to every group. */
int asr_epi_blocks(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, const double* v9, const double* chi, int ngroup,
                   const double* z, int nz, int tail, int precision, int project, double* x, int* mused);

/* Batch-shape autotuner (no counterpart in the reference, which has no device): times the chains of the given groups
 * (depth capped at `levels`, at most 64 of the energies) over tiles per batch {4, 8, 16, 32} and nodes per warp
 * {1, 2, 4, 8} and keeps the fastest shape (a candidate must beat the built-in default, 16 tiles in FP64 and 8 in FP32
 * at 4 nodes per warp, by 3 %) on the operator for this precision; later calls that leave the shape
 * automatic use it.  The shape does not change results beyond the order of the per-block partial sums (rounding).
 * Each candidate is timed on the device (CUDA events around its batches, allocations excluded, best of two runs).
 * At the chosen shape it then times the step kernel with fixed-offset link gathers (links whose orbital operation keeps
 * the orbital order read their nine rows without index decoding; the same bits) against the general one and keeps it
 * when it is 3 % faster.
 * tpb, npw: the chosen shape; times(8) the device times in ms (-1: skipped) or NULL. */
int asr_autotune(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const double* z, int nz, int precision,
                 int levels, int* tpb, int* npw, double* times);

/* The operator's tuned state for a precision: tpb, npw (0: never tuned, the built-in defaults apply), link = 1 when the
 * fixed-offset link gathers are in use, ms(2) the device times of the general and the fixed-offset step at the tuned shape
 * (-1: not timed).  Any pointer may be NULL.  No counterpart in the reference. */
int asr_op_tuning(const asr_op* op, int precision, int* tpb, int* npw, int* link, double* ms);
/* Set the tuned state for a precision (a shape saved from an earlier asr_autotune, or a pinned one): tpb in {4, 8, 16, 32}
 * or 0 (built-in default), npw in {1, 2, 4, 8} or 0, link 0 (general gathers) or 1 (fixed-offset).  Results do not depend
 * on link; the shape changes only the order of the per-block partial sums. */
int asr_op_set_tuning(asr_op* op, int precision, int tpb, int npw, int link);

/* ---- route ed3 (src/asr_ed3.f90): chains on z - K'(z), K' = et - h' + u h' + h' u - h' Qt h', h' = g + d S d ---------- */
typedef struct asr_ed3_group {
  const double *g, *d;                    /* (9, nsp): h' of ed3_setup (:57-79): g = (D_c / D_s)(C - E_nu), d = D_c^1/2 */
  const double *dc, *del, *enu, *o, *p;   /* ed3_t (:24-28): D_c (9); D_s, E_nu,s, o_s, p_s (9, nsp) */
  int central;                            /* species frozen on the start site */
  int start_orb;                          /* 1..9, one dimensional under the group */
  int nlev;                               /* chain depth */
  int reserved;
} asr_ed3_group;
/* ed3_blocks (src/asr_ed3.f90:242-265) of every group at every energy: bk(4, nz, ngroup) complex = G_11, (hG)_11,
 * (hGh)_11 and q1 of the |a> chain minus q1 of the |v> chain; mused(2, nz, ngroup) the depths of the |a> and |v> chains;
 * a, b, c (nlevmax, 2, nz, ngroup) complex chain coefficients and projections, or NULL.  depth_tol > 0: the depth test
 * on g and f of :173-179; tail as asr_chains_run (a closed chain uses the exact fraction, cf_closed :221-236). */
int asr_ed3_blocks(asr_ctx* ctx, asr_op* op, const asr_ed3_group* groups, int ngroup, const double* z, int nz, double depth_tol,
                   int tail, int precision, int project, double* bk, int* mused, double* a, double* b, double* c);

/* Reverse mode of the batched energy-dependent chains (edc route, o = 0, fixed depth nlev per group): g(nz, ngroup) as
 * asr_chains_run, and grad(9, nsp, 3, ngroup) complex = sum_j w(j, q) dG(j, q)/dpar for the parameter arrays of group q:
 * kind 0 the diagonal c (the same derivative applies to e and pb, which enter only as c + e + pb when o = 0), kind 1 d,
 * kind 2 pa.  w(nz, ngroup) complex seeds.  The entries are symmetrised over the orbits of the orbitals under the
 * operator's point group (the group-reduced operator represents only parameters constant on each orbit): derivatives
 * along every group-invariant direction (per l, per orbit) are exact.  stride > 0: the Lanczos vectors are kept every
 * `stride` levels and recomputed in between; stride = 0: every level's vectors are kept when a batch of 4 tiles fits in
 * half the free device memory (no recomputation), else every ceil(sqrt(depth)) levels.  Both give the same bits.  Every tail (none, hull, bp, avg2).  Groups with o != 0 are refused
 * (asr_chains_adjoint_ext).  No counterpart in the reference (gradients of the chain with respect to the species
 * parameters of src/asr_edc.f90:41-71). */
int asr_chains_adjoint(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const double* z, int nz,
                       const double* w, int tail, int precision, int project, int stride, double* g, double* grad);

/* asr_chains_adjoint for the reference's whole operator form: H = E_nu + h - h o h + X(z) with o != 0 (edc_setup's
 * o = o_l D_s / D_c, src/asr_edc.f90:66), chains stopped by the depth test of src/asr_edc.f90:121-127 when
 * depth_tol > 0 (the derivative of the chain at the depth it stopped at, mused(nz, ngroup) optional), and every tail
 * (the Beer-Pettifor fixed point differentiated implicitly).  grad(9, nsp, 5, ngroup) complex, kinds 0 c, 1 d, 2 pa,
 * 3 o, 4 e (pb enters as e does).  No counterpart in the reference. */
int asr_chains_adjoint_ext(asr_ctx* ctx, asr_op* op, const asr_chain_group* groups, int ngroup, const double* z, int nz,
                           const double* w, double depth_tol, int tail, int precision, int project, int stride, double* g,
                           int* mused, double* grad);

/* cf_species (src/asr_chain.f90:67-167) for nchain complex chains a, b (ld, nchain), depth m(nchain), at the energies
 * z(nz, nchain): g(nz, nchain).  edges (optional, (2, nz, nchain)) returns the tail (centre, quarter width). */
int asr_cf_eval(asr_ctx* ctx, const double* a, const double* b, const int* m, int ld, int nchain, const double* z, int nz,
                int tail, double* g, double* edges, int64_t* nfall);

/* asr_cf_eval without device allocation (no edges), for callers that may not call cudaMalloc / cudaFree (they
 * synchronise the device, or device memory belongs to another allocator).  No counterpart in the reference.  The
 * operands go through one static device array of ASR_CF_NOALLOC_BYTES per device; calls whose operands need more
 * (32 ld nchain + 32 nz nchain + 4 nchain + 4 bytes, each part rounded up to 256) return ASR_EINVAL.  The call is
 * synchronous: it copies the operands from host memory and returns after g and nfall are back on the host.  The first
 * call on a context resolves the array's device address and keeps it with the context; make that first call before any
 * stream capture on the device.  Calls that overlap in time on one device share the array and race: serialise them. */
#define ASR_CF_NOALLOC_BYTES (8u << 20)
int asr_cf_eval_noalloc(asr_ctx* ctx, const double* a, const double* b, const int* m, int ld, int nchain, const double* z,
                        int nz, int tail, double* g, int64_t* nfall);

/* reverse mode of cf_species for one chain (host): abar(m), bbar(m) complex receive w dG/da_k and w dG/db_k; g = G.
 * Tails none, hull, bp, avg2; the Beer-Pettifor fixed point is differentiated implicitly (through the sensitivities of
 * the two shifted extreme eigenvalues); a fixed point that did not converge falls back to the hull, as the forward does.
 * No counterpart in the reference. */
int asr_cf_adjoint(const double* a, const double* b, int m, double zr, double zi, int tail, double wr, double wi, double* abar,
                   double* bbar, double* g);

/* ---- KPM on an explicit supercell: kpm_moments / kpm_dos (src/reference/asr_kpm.f90:39-87) on the realisation operator
 *      lmto_real_op (src/reference/asr_lmto_realization.f90:14-191), n species ------------------------------------------- */
typedef struct asr_supercell asr_supercell;
/* nbr(nslot, nsite) 1-based neighbour of every slot, spc(nsite) species 1..nsp, c/d/o/e(9, nsp), block(9, 9, nslot),
 * block0(9, 9) (NULL: zero).  H = E_nu + h - h o h, h = c + d S d, per site by its species (build_lmto_ordered :49-77). */
int asr_supercell_build(asr_ctx* ctx, int nsite, int nslot, const int* nbr, const int* spc, int nsp, const double* c,
                        const double* d, const double* o, const double* e, const double* block, const double* block0,
                        asr_supercell** sc);
int asr_supercell_free(asr_supercell* sc);
/* real_apply (:149-191): y = H x for nvec real vectors x(9 nsite, nvec) */
int asr_supercell_apply(asr_supercell* sc, const double* x, double* y, int nvec);
/* mu(0:nmom-1) = (1/nvec) sum_r <r|T_n((H - cen)/sc)|r> / dim over the Rademacher vectors v0 .. v0+nvec-1 of the
 * counter-based generator (entry q of vector v is +1 iff bit 63 of splitmix64(seed * 0x9E3779B97F4A7C15 + (v << 40) + q)
 * is clear); precision ASR_FP32: FP32 matvec and vectors, FP64 moments.  doubling = 1 takes two moments per matvec. */
int asr_kpm_moments(asr_ctx* ctx, asr_supercell* sc, double cen, double scl, int nmom, int v0, int nvec, uint64_t seed,
                    int precision, int doubling, double* mu);
/* kpm_dos (:68-87), Jackson kernel, host */
int asr_kpm_dos(const double* mu, int nmom, double cen, double scl, const double* e, int ne, double* rho);
/* species layout with first-shell Warren-Cowley order (the role of tools/sqs.py --alpha and tools/sro_closure/sro_mc.c,
 * own swap Monte Carlo): the first z slots of nbr(ldnbr, nsite) are the first shell; alpha(nsp, nsp) unlike-pair targets
 * (NULL: random); spc(nsite) 1-based output; alpha_out(nsp, nsp) the achieved parameters.  Host. */
int asr_sro_layout(int nsite, int z, const int* nbr, int ldnbr, int nsp, const double* conc, const double* alpha,
                   uint64_t seed, int sweeps, int* spc, double* alpha_out);

/* ---- contour (src/asr_contour.f90), host ------------------------------------------------------------------------- */
int asr_gauss_legendre(int n, double* x, double* w);
/* contour_nodes :17-34 (eta_end < 0: to the real axis) */
int asr_contour_nodes(double ebot, double ef, int n, double eta_end, double* z, double* w);
/* contour_nodes_closed :39-58 */
int asr_contour_nodes_closed(double ebot, double ef, double eta, int n_arc, int n_vert, double* z, double* w);
/* contour_nodes_fermi :77-121 (z, w of length 4 + n_main + n_step + 8 + npole) */
int asr_contour_nodes_fermi(double ebot, double mu, double kt, int npole, int n_main, int n_step, double* z, double* w);
/* contour_moment :124-130 */
int asr_contour_moment(const double* z, const double* w, const double* g, int n, double enu, int k, double* m);

#ifdef __cplusplus
}
#endif
#endif
