/*
 * sadmrg.h -- C ABI of the B200 two-site DMRG hot path.
 *
 * Plain C: pointers, sizes and ints; no C++ or torch types.  Every function
 * returns 0 on success or a positive status (SADMRG_ERR_*) and never exits the
 * process.  sadmrg_last_error() gives the message of the last failure.
 *
 * One handle = one CUDA device + one stream; calls on a handle are stream
 * ordered and must come from one host thread at a time.
 *
 * Scalars: real data is double; complex data is interleaved (re, im) double,
 * the layout of std::complex<double>.  Dense blocks are column-major with
 * bond 0 fastest, exactly as the reference's Dense<Scalar>.
 *
 * Reference interfaces replaced (lingwangqs/symmetry-adapted-DMRG-library):
 *   sadmrg_heff_*         DMRG::hamiltonian_vector_multiplication_idmrg   src/dmrg_inst.cpp:283-371
 *                         BlockTensor::hamiltonian_vector_multiplication   src/block_tensor_inst.cpp:2170-2318
 *   sadmrg_heff_lanczos   Lanczos::initialize_lanczos + lanczos1         src/dmrg_inst.cpp:1201-1348
 *   sadmrg_chain_env_update
 *                         DMRG::prepare_site_operator_from_left/right      src/dmrg_inst.cpp:440-695
 *                         (BlockTensor::operator_initial / operator_transformation / operator_pairup /
 *                          overlap_transformation, src/block_tensor_inst.cpp:1283-2167)
 *   sadmrg_svd_truncate   BlockTensor::svd                                 src/block_tensor_inst.cpp:501-637
 *   sadmrg_chain_*        DMRG<Scalar,Sym>::DMRG / do_idmrg / prepare_sweep / sweep / get_enr
 *                                                                           dmrg.hpp:98-131, src/dmrg_inst.cpp:63-943
 */
#ifndef SADMRG_H
#define SADMRG_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sadmrg_handle sadmrg_handle;

enum {
  SADMRG_OK = 0,
  SADMRG_ERR_ARG = 1,
  SADMRG_ERR_CUDA = 2,
  SADMRG_ERR_NOMEM = 3,
  SADMRG_ERR_STATE = 4,
  SADMRG_ERR_NUMERIC = 5,
  SADMRG_ERR_LIMIT = 6,
  SADMRG_ERR_DEVICE_FLAG = 7
};

enum { SADMRG_SYM_U1 = 0, SADMRG_SYM_SU2 = 1 };
enum { SADMRG_PREC_FP64 = 0, SADMRG_PREC_TF32X3 = 1 };

/* A block-sparse tensor (the reference's BlockTensor): bonds with sector
 * labels (U1 charge or SU2 2J) and reduced dimensions, the present blocks by
 * their block index (mixed radix over sector indices, bond 0 fastest), and the
 * present blocks' data concatenated in ascending block-index order. */
typedef struct {
  int nbond;
  int locspin;
  const int* dir;              /* [nbond] */
  const int* nmom;             /* [nbond] sectors per bond */
  const int* q;                /* [sum nmom] sector labels, bond after bond */
  const int* d;                /* [sum nmom] sector dimensions */
  int nblocks;
  const long long* block_index;/* [nblocks], ascending */
  const void* data;            /* all present blocks */
} sadmrg_tensor_desc;

int sadmrg_version(void);
int sadmrg_create(int sym, int cplx, int device, sadmrg_handle** out);
int sadmrg_destroy(sadmrg_handle* h);
const char* sadmrg_last_error(const sadmrg_handle* h);

/* Device status of the tcgen05 GEMM kernels (no counterpart in the reference,
 * whose CPU code has nothing to wait on).  Synchronises the handle's stream,
 * stores 0 if every bounded wait since the last query completed, otherwise a
 * nonzero code (the tiles those waits guarded were left unwritten), and clears
 * it.  The calls that synchronise anyway (heff_apply, heff_lanczos,
 * heff_profile, chain_idmrg, chain_sweep) check it themselves and fail with
 * SADMRG_ERR_CUDA. */
int sadmrg_device_status(sadmrg_handle* h, int* status);
/* Failure-path check of those bounded waits (no counterpart in the reference).
 * Runs one split-precision H_eff*psi of the current plan (on the handle's own
 * zeroed psi buffer) as a single cooperative launch in which the first psi panel
 * set is never reported complete -- its completion target is raised by one for
 * this launch only, a flag nothing sets -- with every wait limited to wait_ns
 * (1 ms .. 2 s).  The items that read those panels give up, their CTAs wait for
 * the copies and MMAs they issued, free their tensor memory and return.  *status
 * is the status word the launch left (nonzero: a wait ran out), which this call
 * clears together with the plan's split-K and dependency counters, so the next
 * call computes normally.  SADMRG_ERR_STATE when the plan has no tcgen05
 * schedule with psi panels. */
int sadmrg_heff_wait_fault_test(sadmrg_handle* h, long long wait_ns, int* status);

/* Lanczos convergence: stop at a check (every 4 steps) once |<v|Hv>|/|Hv| is
 * within ov_tol of 1.  Default 1e-8, the reference's constant (src/dmrg_inst.cpp:1338).
 * The split-precision solver (SADMRG_PREC_TF32X3) applies the same tolerance
 * through the Lanczos residual estimate r = b_m |z_m| (|<v|Hv>|/|Hv| - 1 ~
 * r^2 / (2 E^2)), without check matvecs. */
int sadmrg_set_lanczos_tol(sadmrg_handle* h, double ov_tol);

/* How the split-precision matvec is launched (no counterpart in the reference):
 * 0 psi -> panels, then one tcgen05 launch per stage; 1 the whole matvec as one
 * cooperative launch whose work items wait (bounded) for the panels they read;
 * -1 (default) one launch for plans below 4 GFLOP per matvec (latency bound),
 * one per stage above.  All three give the same bits. */
int sadmrg_set_matvec_fusion(sadmrg_handle* h, int fused);

/* ---- frozen two-site problem: H_eff * psi ---------------------------------
 * ops[] holds every block operator once; term i pairs ops[op1[i]] (left block,
 * legs (a, channel, a')) with ops[op2[i]] (right block, legs (b, channel, b')),
 * the right operators already summed with their couplings as the reference
 * does before calling BlockTensor::hamiltonian_vector_multiplication.
 * hh_left / hh_right may be NULL (null block Hamiltonian).  psi fixes the
 * block structure of every vector passed to apply / lanczos. */
int sadmrg_heff_plan(sadmrg_handle* h, const sadmrg_tensor_desc* psi, const sadmrg_tensor_desc* hh_left,
                     const sadmrg_tensor_desc* hh_right, int nops, const sadmrg_tensor_desc* ops, int nterms,
                     const int* op1, const int* op2);
/* Excited-state penalty of the reference's H_eff (src/dmrg_inst.cpp:352-363):
 * after this call every H_eff*psi (apply, apply_device, apply_noalloc, lanczos)
 * also subtracts sum_k weights[k] <o_k|psi> o_k, with o_k the nvec vectors in
 * vecs_host (psi's layout, one after another; the lower states projected on this
 * two-site basis) and weights[k] their energies (the reference's gs_enr[k]).
 * nvec = 0 removes the penalty.  The per-stage and per-launch profiles and the
 * graph replay time the sector products only. */
int sadmrg_heff_set_penalty(sadmrg_handle* h, int nvec, const void* vecs_host, const double* weights);
/* Autotuning of the split-precision matvec (no counterpart in the reference).
 * With it on (the default) every new H_eff plan times candidate tcgen05
 * schedules on itself -- output tile width 64 or 128, split-K chunks of at
 * least 16 k slabs or none, one cooperative launch or one per stage -- with
 * items capped at 32 k slabs, two CTAs per SM -- with CUDA events on the
 * handle's stream, and keeps the fastest; the choice is
 * cached per block-size histogram of the plan (jobs by log2 of m, n and k) for
 * the life of the process.  Off: fixed heuristics.  The FP64 path is never
 * tuned (its rounding does not depend on a timing). */
int sadmrg_set_autotune(sadmrg_handle* h, int on);
/* QR preconditioning of the block SVD (no counterpart in the reference, whose
 * LAPACK gesvd needs none).  With it the one-sided Jacobi runs on R1^H, where
 * Q R is a Householder QR of a sector block's columns ordered by decreasing
 * norm and Q1 R1 one of R^H (Drmac & Veselic 2008), which cuts its sweeps by
 * about 40%; without it the Jacobi runs on the block itself.  on = 1 (the
 * default): for calls whose widest block has at least 32 columns (below that
 * the QRs cost about what they save); 2: always; 0: never.  The truncation
 * means the same either way: the same singular values and vectors to
 * rounding. */
int sadmrg_set_svd_precondition(sadmrg_handle* h, int on);
/* Block SVD visits (no counterpart in the reference): 0 (the default) keeps a
 * Jacobi visit's columns of W and V in shared memory where the launch's largest
 * pair fits, 1 always streams them in row chunks as for blocks too tall to fit.
 * The same results either way; for tests and profiling. */
int sadmrg_set_svd_stream(sadmrg_handle* h, int on);
/* Block SVD Jacobi column blocks (no counterpart in the reference): 8 or 16
 * columns per block, or 0 (the default) for 8 when the widest round of 16-column
 * pairs would keep fewer than half the SMs busy and 16 otherwise.  The same
 * results either way; for tests and profiling. */
int sadmrg_set_svd_block(sadmrg_handle* h, int b);
/* A fixed tile choice for the H_eff plans made after this call, instead of the
 * autotuner or the heuristics: width 64 or 128 (0 returns to them), fewest slabs
 * per split-K chunk when the tiles cannot fill the GPU (0: no such split), most
 * slabs per item (0: no cap), CTAs per SM (1, or 2 at width 64), one cooperative
 * launch per matvec (1), one per stage (0) or the default rule (-1).  For
 * profiling one schedule. */
int sadmrg_set_tiles(sadmrg_handle* h, int bn, int kc_min, int kc_max, int ctas_per_sm, int one_launch);
/* The current plan's tile choice: out[0] tile width, out[1] fewest slabs per
 * split-K chunk when the tiles cannot fill the GPU (0: no such split), out[2]
 * most slabs per item (0: no cap), out[3] CTAs per SM, out[4] 1 when a matvec is
 * one cooperative launch, out[5] 0 heuristic / 1 timed for this plan / 2 from the
 * cache / 3 set by sadmrg_set_tiles, out[6] the number of candidates timed, then
 * per candidate (width, chunk, cap, CTAs per SM, one launch, ms per matvec).  *n is the number of values; the first min(cap, *n)
 * are written. */
int sadmrg_heff_tiles(sadmrg_handle* h, int cap, double* out, int* n);
/* psi elements, algorithmic flops and bytes of one matvec, number of sector products */
int sadmrg_heff_info(sadmrg_handle* h, long long* n, double* flops, double* bytes, int* ntasks);
/* out = H_eff psi with host buffers (copies in and out on the handle's stream) */
int sadmrg_heff_apply(sadmrg_handle* h, const void* psi_host, void* out_host, int precision);
/* out = H_eff psi with device pointers (no copies) */
int sadmrg_heff_apply_device(sadmrg_handle* h, const void* psi_dev, void* out_dev, int precision);
/* out = H_eff psi with device pointers, allocating nothing.  No counterpart in
 * the reference (its H*v allocates per call).  For callers that cannot allocate
 * device memory when they apply the operator -- a host whose memory pool is
 * capped or fully reserved, or a solver loop that must not touch the allocator
 * between steps.  The plan (sadmrg_heff_plan) must exist already; the stage-0
 * products and split-K partial tiles go to one fixed 32 MiB device array
 * compiled into the library, and a plan that needs more is refused with
 * SADMRG_ERR_LIMIT.  The first call on a device looks that array's device
 * address up (cudaGetSymbolAddress); make it before any stream capture.  Every
 * call shares the array and overwrites it, so calls that overlap on the GPU
 * (two streams, two handles on one device) race. */
int sadmrg_heff_apply_noalloc(sadmrg_handle* h, const void* psi_dev, void* out_dev, int precision);
/* Per-stage device time of one H_eff*psi (CUDA events on the handle's stream,
 * averaged over reps): ms[0] stage 0 (X = op1^T psi products), ms[1] stage 1
 * (the output accumulation lists); flops[] the algorithmic flops of each stage.
 * psi_dev / out_dev may be NULL (the handle's own buffers are used). */
int sadmrg_heff_profile(sadmrg_handle* h, int precision, int reps, const void* psi_dev, void* out_dev, double* ms,
                        double* flops);
/* Per-launch device time of one H_eff*psi (no counterpart in the reference; for
 * rooflines): an event after every kernel the matvec launches, averaged over
 * reps.  On return *nlaunch is the number of launches of one matvec; for the
 * first min(cap, *nlaunch) of them kind[i] says what ran (0 psi -> TF32 panels,
 * 1 + 2*stage: the grouped GEMM of that stage, 2 + 2*stage: its split-K
 * reduction, 5: the whole matvec in one launch) and ms[i] its mean time. */
int sadmrg_heff_launch_profile(sadmrg_handle* h, int precision, int reps, const void* psi_dev, void* out_dev, int cap,
                               int* nlaunch, int* kind, double* ms);
/* The same matvec replayed from a CUDA graph (no counterpart in the reference):
 * one H_eff*psi on (psi_dev, out_dev) is captured once, the graph is launched
 * reps times, and *ms is the mean device time per replay (CUDA events). */
int sadmrg_heff_graph_bench(sadmrg_handle* h, int precision, int reps, const void* psi_dev, void* out_dev,
                            double* ms);
/* Timed steps of the same captured matvec (no counterpart in the reference):
 * the graph of one H_eff*psi on (psi_dev, out_dev) is captured once; then per
 * step, on the handle's stream, the first half of the flush_bytes at flush_dev
 * is overwritten and the second half read (each half larger than the L2, so
 * the operands are evicted and the written lines are back in memory before the
 * step; 0 for none), and the graph is launched between two CUDA events.  ms[i]
 * is the device time of step i (steps values). */
int sadmrg_heff_graph_steps(sadmrg_handle* h, int precision, int steps, const void* psi_dev, void* out_dev,
                            void* flush_dev, long long flush_bytes, double* ms);
/* kernels one H_eff*psi launches at this precision (the penalty's included) */
int sadmrg_heff_launches_per_matvec(sadmrg_handle* h, int precision, int* n);
/* Lanczos ground state (lanczos1) from psi; psi is overwritten by the Ritz vector.
 * precision SADMRG_PREC_TF32X3 runs the split-precision Lanczos followed by an
 * FP64 restart from its result. */
int sadmrg_heff_lanczos(sadmrg_handle* h, void* psi_host, int mlanc, int precision, double* energy, int* matvecs);
/* Lanczos::lanczos2 (src/dmrg_inst.cpp:1352-1397), FP64: the same recurrence
 * without convergence checks -- all mlanc steps; at a breakdown (b < 1e-6 from
 * step 2) the Ritz pair of the steps before it.  psi is overwritten by the Ritz
 * vector. */
int sadmrg_heff_lanczos2(sadmrg_handle* h, void* psi_host, int mlanc, double* energy, int* matvecs);

/* ---- many independent instances, one launch per stage ---------------------
 * No counterpart in the reference (one DMRG per process).  sadmrg_batch_add
 * appends the H_eff plan of another handle `inst` (same device, symmetry and
 * scalar type) to h's batch; the instance handle may be destroyed once it has
 * been added.  sadmrg_batch_finalize merges the plans: instance i's vectors are
 * the segment [offsets[i], offsets[i+1]) of one long vector, and every batched
 * matvec runs all instances' sector products in one launch per stage.
 * sadmrg_batch_lanczos runs lanczos1 (or the mixed solver) on every instance at
 * once from psi_host (all segments), leaves each instance's Ritz vector in its
 * segment and its energy in energies[i]; matvecs[i] counts the matvecs instance i
 * needed, *batched_matvecs the batched launches. */
int sadmrg_batch_add(sadmrg_handle* h, sadmrg_handle* inst);
int sadmrg_batch_finalize(sadmrg_handle* h);
int sadmrg_batch_clear(sadmrg_handle* h);
int sadmrg_batch_info(sadmrg_handle* h, int* ninst, long long* n, double* flops, int cap, long long* offsets);
int sadmrg_batch_apply(sadmrg_handle* h, const void* psi_host, void* out_host, int precision);
int sadmrg_batch_lanczos(sadmrg_handle* h, void* psi_host, int mlanc, int precision, double* energies, int* matvecs,
                         int* batched_matvecs);
/* mean device time (ms, CUDA events, back to back) of one batched matvec over reps */
int sadmrg_batch_profile(sadmrg_handle* h, int precision, int reps, double* ms);

/* ---- block SVD truncation ---------------------------------------------------
 * psi: 2-leg two-site vector.  tu / tv: the current site tensors (only their
 * bonds 0 and 1 are read).  p1 / p2: powers of the singular values absorbed
 * into U / V.  The new site tensors are staged and read with sadmrg_staged_*
 * (which = 0 for U, 1 for V). */
int sadmrg_svd_truncate(sadmrg_handle* h, const sadmrg_tensor_desc* psi, const sadmrg_tensor_desc* tu,
                        const sadmrg_tensor_desc* tv, double p1, double p2, int max_dcut, int* kept,
                        double* discarded_weight);

/* ---- chain driver (DMRG<Scalar,Sym>) ---------------------------------------
 * lx, ly: lattice as the reference's DMRG(xx, yy, ...) constructor (a chain of
 * L sites is lx = 1, ly = L); open = 1 drops the periodic wrap; J2 adds
 * next-nearest-neighbour couplings along the site order. */
int sadmrg_chain_create(sadmrg_handle* h, int lx, int ly, int bondd, int physpn, int totspin, int open, double J2);
/* Adds Dz (S_a x S_b)_z on every J1 bond a < b (chain order) of a U(1) complex
 * chain: the bond's S+_a S-_b and S-_a S+_b parts get (J + i Dz)/2 and
 * (J - i Dz)/2.  Call before sadmrg_chain_idmrg / sadmrg_chain_read_mps.  No
 * counterpart in the reference (one real coupling per pair, coup[] in
 * src/dmrg_inst.cpp:146-160); SADMRG_ERR_ARG for SU(2) or real scalars. */
int sadmrg_chain_set_dm(sadmrg_handle* h, double dz);
/* The chain targets excited state exci (the max_exci argument of the reference's
 * DMRG constructor, src/dmrg_inst.cpp:64-112).  Call before sadmrg_chain_read_mps,
 * which then reads this state's files (index exci) and, as DMRG::read_mps(read1,
 * read2) (:1081-1140), the lower states 0 .. exci-1 and the last energy of each
 * (enr-<ns>-<D>-<2S>-<idx>.dat); the sweeps keep their overlap environments
 * (:440-583, 862-868), project them on every two-site basis (:412-437) and add
 * the penalty -E_j <o_j|psi> o_j to H_eff*psi (:352-363).  U(1) and SU(2);
 * an excited state starts from read_mps, not iDMRG.
 * Checkpoint, ww and enr files carry the state's index. */
int sadmrg_chain_set_excited(sadmrg_handle* h, int exci);
int sadmrg_chain_set_precision(sadmrg_handle* h, int precision);
int sadmrg_chain_idmrg(sadmrg_handle* h, double* energy);
int sadmrg_chain_prepare_sweep(sadmrg_handle* h);
int sadmrg_chain_sweep(sadmrg_handle* h, double* energy);
/* DMRG::read_mps(bond_read) / save_mps2 checkpoint files (src/dmrg_inst.cpp:947-1079):
 * uu-<ns>-<D>-<2S>-<exci>-<site>.dat (bond structure, text) and .bin (block data,
 * then SU(2) CGC blocks) in directory dir, exci = 0 but for an excited-state chain
 * (sadmrg_chain_set_excited).  read_mps is followed by prepare_sweep. */
int sadmrg_chain_read_mps(sadmrg_handle* h, const char* dir, int bond_read);
int sadmrg_chain_save_mps(sadmrg_handle* h, const char* dir);
/* DMRG::save_ww / read_ww (src/dmrg_inst.cpp:1145-1165): the singular values of
 * the truncations.  The chain keeps them as the reference's ww array: every
 * truncation overwrites its first n entries (the kept values sector by sector,
 * then from position kept the discarded ones) and the return pass of a sweep
 * clears the first bondd entries before each truncation (src/dmrg_inst.cpp:934).
 * save_ww writes bondd * (physpn + 1) doubles to ww-<ns>-<D>-<2S>-0.bin in dir;
 * read_ww reads the first bond_read doubles of ww-<ns>-<bond_read>-<2S>-0.bin,
 * or sets them to 1 when that file is absent. */
int sadmrg_chain_save_ww(sadmrg_handle* h, const char* dir);
int sadmrg_chain_read_ww(sadmrg_handle* h, const char* dir, int bond_read);
/* DMRG::save_enr / read_enr (src/dmrg_inst.cpp:993-1016): save_enr appends the
 * chain's energy (16 significant digits) to enr-<ns>-<D>-<2S>-0.dat in dir;
 * read_enr sets it to the last value of enr-<ns>-<bond_read>-<2S>-0.dat (unchanged
 * when the file is absent). */
int sadmrg_chain_save_enr(sadmrg_handle* h, const char* dir);
int sadmrg_chain_read_enr(sadmrg_handle* h, const char* dir, int bond_read);
/* the chain's ww array: *n its length, the first min(cap, *n) values to out */
int sadmrg_chain_ww(sadmrg_handle* h, int cap, int* n, double* out);
/* Lanczos length of the chain's solves: the reference's constant mlanc = 40
 * (src/dmrg_inst.cpp:267), capped like it at the vector length + 1.  The stop
 * test is sadmrg_set_lanczos_tol. */
int sadmrg_chain_set_mlanc(sadmrg_handle* h, int mlanc);
/* Freeze the two-site problem at bond (il, il+1): psi = the current site tensors'
 * product (DMRG::prepare_input_vector), the fused environments and the H_eff plan
 * become the handle's heff plan (sadmrg_heff_*), psi is staged (which = 0).  If
 * export_dir is not NULL or empty the problem is also written there, one
 * <name>.txt (bonds and present blocks) + <name>.bin (data) pair per tensor. */
int sadmrg_chain_freeze(sadmrg_handle* h, int il, const char* export_dir);
/* sectors of bond 2 of site tensor uu[site]: labels and dimensions */
int sadmrg_chain_bond(sadmrg_handle* h, int site, int cap, int* nsec, int* q, int* d);
/* timers: [lanczos_s, env_s, svd_s, prep_s, matvecs, heff_flops, gemm_flops, launches, discarded,
 *          near_ties (truncations whose cut split a pair of singular values equal to 1e-8, or
 *          whose per-sector 1e-10 relative cut-off met a value within two decades of it),
 *          svd_kernel_s (device time of the Jacobi sweeps), svd_sweeps,
 *          plan_s (host time of building H_eff plans, part of lanczos_s),
 *          stop_ties (truncations whose cut gap -- D-th minus (D+1)-th singular value over
 *          |psi| -- is below 10 sqrt(Lanczos ov_tol): the stop test fixes psi only to about
 *          that, so two correct runs may cut such a bond differently)]; the first n are written */
int sadmrg_chain_stats(sadmrg_handle* h, double* out, int n);
/* Per bond (index il of its two-site pair (il, il + 1)), what its last truncation
 * flagged: 1 a rounding tie (as near_ties), 2 a stop-test tie (as stop_ties);
 * flags[i] for i < cap. */
int sadmrg_chain_bond_flags(sadmrg_handle* h, int cap, int* flags);
/* kind: 0 = uu[site], 1 = hh[site], 2 = opr[site][k] */
int sadmrg_chain_set_tensor(sadmrg_handle* h, int kind, int site, int k, const sadmrg_tensor_desc* t);
int sadmrg_chain_stage_tensor(sadmrg_handle* h, int kind, int site, int k);
/* prepare_site_operator_from_left (dir = 0) / from_right (dir = 1);
 * real_env = 1: with uu[site] itself; 0: in the fused (block x site) basis */
int sadmrg_chain_env_update(sadmrg_handle* h, int site, int dir, int real_env);

/* ---- staged tensors (results) ----------------------------------------------- */
int sadmrg_staged_info(sadmrg_handle* h, int which, int* nbond, int* locspin, int* nsectors, int* nblocks,
                       long long* nelem);
int sadmrg_staged_read(sadmrg_handle* h, int which, int* dir, int* nmom, int* q, int* d, long long* block_index,
                       void* data);

#ifdef __cplusplus
}
#endif
#endif /* SADMRG_H */
