// kernels.cuh -- device task formats and launchers.
//
// Every contraction on the hot path (H_eff*psi, environment updates, the
// projector products after the SVD) is lowered on the host to a list of dense
// sector GEMMs; one launch executes a whole list.  Operands are addressed as
// (base buffer id, element offset) so a plan built once per bond can be run on
// any psi / output vector by swapping base pointers.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

namespace sadmrg {

enum TermFlags : int { TF_TA = 1, TF_CA = 2, TF_TB = 4, TF_CB = 8 };
enum JobFlags : int { JF_ACCUM = 1 };   // C += sum(terms); otherwise C = sum(terms)
enum Precision : int { PREC_FP64 = 0, PREC_TF32X3 = 1 };
constexpr int kMaxBases = 8;

struct GemmTerm {             // alpha * op(A) * op(B), A: m x k, B: k x n after op
  long long aoff, boff;       // element offsets (elements of the scalar type)
  int abuf, bbuf;             // base buffer ids
  int lda, ldb, k, flags;
  double ar, ai;              // alpha (imaginary part ignored for real data)
};
struct GemmJob {              // C (m x n, column-major, ldc) receives its terms
  long long coff;
  int cbuf, m, n, ldc;
  int t0, nt, flags;
  int tag;                    // instance of a merged batch plan (0 otherwise): a launch given a mask
                              // skips every item of a job whose mask[tag] is 0
};
struct GemmTile {
  int job, tm, tn;
};
struct WorkItem {             // one output tile x a contiguous range of the job's concatenated k
  int job, tm, tn;
  int t0, k0, kcount;         // first term (relative to the job's t0), offset in it, total k
  int slot;                   // < 0: write C directly; otherwise the partial-tile slot
  int red;                    // split items: their tile's RedItem
};
struct RedItem {              // C tile = sum of slots [slot0, slot0 + nslot) (fixed order)
  int job, tm, tn, slot0, nslot;
};
struct Bases {
  void* p[kMaxBases];
};


// Grouped GEMM over work items (deterministic split-K; see gemm.cu).
// Split items write partial tiles; the last of a tile's items sums them (tile_cnt
// holds one zeroed counter per RedItem and is left zeroed).
// mask: null, or per job tag; items of a job with mask[tag] == 0 do nothing.
void launch_items(bool cplx, int prec, const GemmTerm* terms, const GemmJob* jobs, const WorkItem* items, int nitems,
                  const Bases& b, void* work, const RedItem* reds, int* tile_cnt, const int* mask, cudaStream_t s);

// ---- tcgen05 3xTF32 over TF32 hi/lo operand panels (umma.cu) --------------
// An operand (rows x K after op) is stored as panels: panel (p, s) holds rows
// [p*T, p*T + T) and k [32 s, 32 s + 32) as a hi plane then a lo plane, each
// [kg = 0..7][row = 0..T-1][4 consecutive k] of TF32 bit patterns (x ~ hi + lo),
// zero padded; it starts at dst + (p * nslab + s) * T * 256 bytes.  This is the
// K-major, no-swizzle core-matrix layout tcgen05.mma reads, so a panel moves
// into shared memory as one contiguous bulk copy.
// Complex products run as real ones of twice the size: C = A B (complex m x n,
// k) is Ch = Ah Bh with Ch (2m x n) and Bh (2k x n) the interleaved storage of
// C and B read as real column-major matrices (no copy), and Ah (2m x 2k) the
// real form of A, Ah(2i+p, 2j+q) = Re A(i,j) for p == q, -Im A(i,j) for
// (p, q) = (0, 1), Im A(i,j) for (1, 0).  The real flop count is the complex
// one (8 per complex multiply-add), and the pack kernel writes Ah / Bh panels
// straight from the complex operands (cmode 1 / 2).
constexpr int kPanelK = 32;
constexpr int kUmmaTileM = 128;
struct PackJob {              // FP64 matrix -> panels
  long long src;              // element offset in its source buffer
  long long dst;              // byte offset of panel (0, 0) in the packed buffer
  long long chunk0;           // first 16-byte chunk of this job in the launch (a multiple of 256)
  int srcbuf, ld, rows, K, trans, T;   // trans 0: (r, k) at src[r + k*ld]; 1: at src[k + r*ld]
  int cmode;                  // 0 real; complex source (src, ld in complex elements, rows / K of the real
                              // form): 1 Ah (rows 2m, K 2k), 2 Bh read as rows n x K 2k
  int conj;                   // complex: conjugate the source elements first
  int sparse;                 // 1: chunks of the real rows and k only (the padding of the
                              // panels is zero already and never written), 0: whole panels
};
struct UTerm {                // a term's operands as panel sets: A (T = 128), B (T = BN)
  long long a, b;             // byte offsets of panel (0, 0)
  int abuf, bbuf;             // 0: constant panels, 1: per-apply panels
  int nslab, klast;           // k slabs, k of the last slab (1..32)
  int adep, bdep;             // dependency counter of the A / B panels written in the same launch, or -1
};
struct UJob {                 // output tile grid of one job
  long long coff;             // FP64 output: bases.p[cbuf] + coff, column-major, ldc
  long long pack;             // >= 0: the result becomes A panels (T = 128) at this byte offset of the
                              // per-apply buffer, scaled by alpha, with pack_nslab slabs per panel
  double alpha;
  int cbuf, m, n, ldc, flags, t0, nt, pack_nslab;
  int dep;                    // counter bumped per finished tile (results read as panels later), or -1
  int tag;                    // as GemmJob::tag
  int cx;                     // complex plan: the tile is a real-form block (rows 2i, 2i+1 = Re, Im of
                              // row i); panels of the result are written in the real form Xh (cmode 1)
};
struct UItem {                // one output tile x a run of consecutive slabs
  int job, tm, tn, t0, s0, nslab, slot;   // t0: first term (absolute), s0: its first slab; slot < 0: direct
  int red;                    // split items: their tile's URed
};
struct URed {                 // C tile = sum of FP32 partial slots [slot0, slot0 + nslot) in fixed order
  int job, tm, tn, slot0, nslot;
};
struct UBufs {
  const unsigned char* pconst;
  unsigned char* pvar;
  float* slots;
  int* tile_cnt;              // per URed: items of the tile finished in this launch (reset by the last)
  int* deps;                  // dependency counters (psi pack jobs, then stage-0 results), zero between launches
  const int* dep_target;      // value each counter reaches once its panels are complete
  unsigned* fin;              // CTAs finished (the last one clears deps)
  const int* mask;            // null, or per job tag: 0 skips the job's items (not with wait_deps)
};
constexpr int kMaxPackJobs = 1024;   // psi pack jobs one fused launch can count
struct UPhase {               // what one launch does besides its items
  const PackJob* pk;          // psi -> panels jobs packed at the start of the launch
  const int* pk_blk;          // pack block (256 chunks) -> job
  int npk_blocks;             // 0: no packing in this launch
  int npk_jobs;
  int wait_deps;              // items wait for panels written in this launch (cooperative launch)
  int ndeps;
  long long wait_ns;          // limit of every bounded wait; 0: the default (2 s)
  int ctas_per_sm;            // 2: two CTAs per SM, each with a 2-stage ring (tile width 64 only); else one
};
// one 256-thread block per 256 chunks; blk_job[block] = its job
void launch_pack(const PackJob* jobs, const int* blk_job, int nblocks, const Bases& b, unsigned char* dst,
                 cudaStream_t s);
// One launch of the tcgen05 executor: optional psi packing, then the items.  With
// ph.wait_deps the whole matvec (pack, stage 0, stage 1) runs as one cooperative
// launch, every item waiting (bounded) for the panels it reads.
void launch_umma_items(int bn, const UTerm* terms, const UJob* jobs, const UItem* items, const URed* reds, int nitems,
                       const Bases& b, const UBufs& u, const UPhase& ph, cudaStream_t s);
// status word of the tcgen05 kernels: 0 = fine, otherwise a bounded wait ran out
// (the tiles it guarded were not written); reset clears it.  -1 if unreadable.
int umma_status(bool reset);
int device_sm_count();
constexpr int kMaxDevices = 64;
// cudaFuncSetAttribute(fn, MaxDynamicSharedMemorySize, bytes) once per device
// (the attribute is per device); done[] holds one flag per device ordinal
void ensure_smem_attr(const void* fn, int bytes, unsigned char* done);
// Fixed device scratch of the allocation-free H_eff*psi entry point (gemm.cu).
constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;
// Device address of that scratch on the current device (looked up once per
// device); returns 0 or a cudaError_t value.
int noalloc_scratch(void** ptr);
int gemm_tile_m(bool cplx, int prec);
int gemm_tile_n(bool cplx, int prec);

// ---- block utilities -------------------------------------------------------
struct Seg {                  // y[doff + i] (+)= alpha * x[soff + i], i < n
  long long doff, soff;
  long long n;
  double ar, ai;
};
void launch_seg_axpy(bool cplx, void* y, const void* x, const Seg* segs, int nseg, cudaStream_t s);

struct Transp {               // dst (cols x rows) = src (rows x cols)^T
  long long soff, doff;
  int rows, cols;
};
void launch_block_transpose(bool cplx, void* dst, const void* src, const Transp* t, int nt, cudaStream_t s);

struct Perm3 {                // dst block = src block (d0 x d1 x d2, column-major) with its legs
  long long soff, doff;       // permuted: leg k of dst is leg p[k] of src
  int d[3], p[3];
};
void launch_permute3(bool cplx, void* dst, const void* src, const Perm3* t, int nt, cudaStream_t s);

struct FuseFill {             // identity embedding of a fuse block (d0,d1,d2): 1 at (a,b,pos+b*d0+a)
  long long off;
  int d0, d1, d2, pos;
};
void launch_fuse_fill(bool cplx, void* data, const FuseFill* f, int nf, cudaStream_t s);

struct Gather {               // dst (rows x kept) = src[rows, perm[c]] * w[c]^p  (optionally conjugated)
  long long soff, doff;       // soff: first row of the source column block (column 0)
  int lds, rows, kept, conj;
  long long woff;             // sorted singular values (double) offset
  long long poff;             // offset into the column permutation
  double p;                   // exponent applied to singular values (0 => none)
};
void launch_gather(bool cplx, void* dst, const void* src, const double* w, const int* perm, const Gather* g, int ng,
                   cudaStream_t s);
// x *= alpha (host scalar)
void launch_scale(bool cplx, void* x, double ar, double ai, long long n, cudaStream_t s);
// read bytes (a multiple of 16) of x and discard them (sink: a device word, written
// only by an unlikely data pattern)
void launch_read(const void* x, long long bytes, unsigned* sink, cudaStream_t s);
// fill with a constant
void launch_fill(bool cplx, void* x, double vr, double vi, long long n, cudaStream_t s);

// ---- Krylov vector operations ---------------------------------------------
// out[j] = <V_j | x> (conjugated first argument), j < nv, deterministic, one launch
// (counter: a device word, zero between launches).  scalar_op >= 0 also applies a
// Krylov scalar step to out[0] in the same launch: 0 -> scalar_out[0] =
// beta_prev[0], scalar_out[1] = Re out[0] (three-term recurrence coefficients);
// 1 -> scalar_out[0] = sqrt(|Re out[0]|) (a norm).
void launch_multi_dot(bool cplx, const void* V, long long ldv, int nv, const void* x, long long n,
                      double* partial, int npart, void* out, unsigned* counter, cudaStream_t s, int scalar_op = -1,
                      const double* beta_prev = nullptr, void* scalar_out = nullptr);
// x -= sum_j c[j] V_j   (c read from device memory)
void launch_multi_axpy(bool cplx, void* x, const void* V, long long ldv, int nv, const void* c, long long n,
                       cudaStream_t s);
// x *= 1 / scal[0].  scal is a device double.
void launch_scale_inv(bool cplx, void* x, const double* scal, long long n, cudaStream_t s);
// y = sum_j c[j] V_j (host coefficients, real)
void launch_lincomb(bool cplx, void* y, const void* V, long long ldv, int nv, const double* c_dev, long long n,
                    cudaStream_t s);

// ---- segmented Krylov operations (independent instances back to back) -----
// segment s covers [seg[s], seg[s + 1]) of every vector; one block per segment
// out[s * nv + j] = <V_j | x> on segment s
void launch_seg_multi_dot(bool cplx, const void* V, long long ldv, int nv, const void* x, const long long* seg,
                          int nseg, void* out, cudaStream_t s);
// x -= sum_j c[s * cstride + j] V_j on segment s
void launch_seg_multi_axpy(bool cplx, void* x, const void* V, long long ldv, int nv, const void* c, int cstride,
                           const long long* seg, int nseg, cudaStream_t s);
// x *= scal[s * sstride] (inv = 0) or 1 / scal[s * sstride] (inv = 1) on segment s
void launch_seg_scale(bool cplx, void* x, const double* scal, int sstride, int inv, const long long* seg, int nseg,
                      cudaStream_t s);
// y = sum_j c[s * cstride + j] V_j (real c) on the segments with mask[s] != 0
void launch_seg_lincomb(bool cplx, void* y, const void* V, long long ldv, int nv, const double* c, int cstride,
                        const int* mask, const long long* seg, int nseg, cudaStream_t s);
// per segment: op 0: coef[2s] = beta_prev[s * bstride], coef[2s + 1] = Re(dot[s]); op 1: out[s * ostride] =
// sqrt(|Re dot[s]|)
void launch_seg_lanczos_scalar(bool cplx, int op, const void* dot, const double* beta_prev, int bstride, void* out,
                               int ostride, int nseg, cudaStream_t s);

// ---- one-sided Jacobi SVD of sector blocks --------------------------------
struct SvdJob {
  long long aoff;             // input block (m x n, lda = m) in the input buffer
  long long woff;             // work: max(m,n) x min(m,n) columns being orthogonalised
  long long voff;             // accumulated rotations: min(m,n) x min(m,n)
  long long soff;             // singular values (double), min(m,n)
  int m, n, trans;            // trans = 1 when m < n (work on A^H)
};
// Host driver: one launch per round of block pairs, one sync per sweep to test
// convergence.  Returns the sweeps taken, or -1 if max_sweeps was reached.
// kernel_ms (optional): device time of the sweep kernel when it ran as one launch
// (with the QR preconditioning: plus the QR and the Q application).
// precondition: Jacobi on R1^H after Householder QRs of the norm-ordered columns
// and of R^H (fewer sweeps): 0 never, 1 when the widest block has at least 32
// columns, 2 always; the outputs have the same meaning either way.
// stream: 1 streams every visit's rows in chunks even where the pair's columns
// would fit in shared memory (same results; covers that path on small problems).
// block: Jacobi column blocks of 8 or 16, 0 for the rule (8 when the widest round
// of 16-column pairs would keep fewer than half the SMs busy).
int run_jacobi_svd(bool cplx, const void* a, void* work, void* vmat, double* sv, const std::vector<SvdJob>& jobs,
                   int max_sweeps, cudaStream_t s, double* kernel_ms = nullptr, int precondition = 1,
                   int stream = 0, int block = 0);

}  // namespace sadmrg
