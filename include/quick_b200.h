/*
 * quick_b200.h -- C ABI of the B200-native two-electron Fock build ("get2e").
 *
 * Two layers share one implementation:
 *
 * 1. Drop-in entry points with the names, argument order and by-reference
 *    calling convention of QUICK's own GPU shim (gfortran-style trailing
 *    underscore), so QUICK's unchanged Fortran SCF driver links against this
 *    library instead of the reference's get2e.  They act on one process-wide
 *    default context, exactly like the reference's global `gpu` object
 *    (src/gpu/cuda/gpu_type.h:512).  Like the reference they return no status
 *    (except where the reference has an `ierr`); `qk_last_status()` reports
 *    the most recent failure.
 *
 * 2. A context API (`qk_*`) with explicit handles, status returns, device
 *    pointers and CUDA streams, for callers that batch several molecules or
 *    keep data resident on the GPU.
 *
 * Array conventions on the drop-in layer are QUICK's: Fortran column-major,
 * 1-based index values, MAXPRIM rows in gccoeff/gcexpo (20, the f-enabled
 * build; see qk_set_maxprim).  No torch types appear anywhere in this ABI.
 */
#ifndef QUICK_B200_H
#define QUICK_B200_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- statuses */
enum {
    QK_OK = 0,
    QK_ERR_NO_DEVICE = 24,        /* same code as gpu_init_device_ (src/gpu/cuda/gpu.cu:291-330) */
    QK_ERR_INVALID_ARG = 101,
    QK_ERR_NOT_READY = 102,       /* a required upload has not happened yet */
    QK_ERR_CUDA = 103,
    QK_ERR_OUT_OF_MEMORY = 104,
    QK_ERR_UNSUPPORTED = 105,     /* e.g. angular momentum above the compiled maximum */
    QK_ERR_BASIS_LAYOUT = 106     /* KLMN / cons do not follow QUICK's convention */
};

/* ======================================================= drop-in entry points */

/* replaces gpu_new_ (src/gpu/cuda/gpu.cu:197) */
void gpu_new_(int *ierr);
/* replaces gpu_set_device_ (src/gpu/cuda/gpu.h:14) */
void gpu_set_device_(int *gpuid, int *ierr);
/* replaces gpu_init_device_ (src/gpu/cuda/gpu.cu:281) */
void gpu_init_device_(int *ierr);
/* replaces gpu_allocate_scratch_ (src/gpu/cuda/gpu.cu:437); nothing to allocate here */
void gpu_allocate_scratch_(bool *allocate_gradient_scratch);
/* replaces gpu_deallocate_scratch_ (src/gpu/cuda/gpu.cu:496) */
void gpu_deallocate_scratch_(bool *deallocate_gradient_scratch);
/* replaces gpu_setup_ (src/gpu/cuda/gpu.cu:539) */
void gpu_setup_(int *natom, int *nbasis, int *nElec, int *imult, int *molchg, int *iAtomType);
/* replaces gpu_upload_method_ (src/gpu/cuda/gpu.cu:722); only HF (method 0) has exchange 1.0 */
void gpu_upload_method_(int *quick_method, bool *is_oshell, double *hyb_coeff);
/* replaces gpu_upload_xyz_ (src/gpu/cuda/gpu.cu:776); xyz(3,natom) in Bohr */
void gpu_upload_xyz_(double *atom_xyz);
/* replaces gpu_upload_atom_and_chg_ (src/gpu/cuda/gpu.cu:820) */
void gpu_upload_atom_and_chg_(int *atom, double *atom_chg);
/* replaces gpu_upload_basis_ (src/gpu/cuda/gpu.cu:1782), same 29 arguments */
void gpu_upload_basis_(int *nshell, int *nprim, int *jshell, int *jbasis, int *maxcontract,
                       int *ncontract, int *itype, double *aexp, double *dcoeff,
                       int *first_basis_function, int *last_basis_function,
                       int *first_shell_basis_function, int *last_shell_basis_function,
                       int *ncenter, int *kstart, int *katom, int *ktype, int *kprim, int *kshell,
                       int *Ksumtype, int *Qnumber, int *Qstart, int *Qfinal, int *Qsbasis,
                       int *Qfbasis, double *gccoeff, double *cons, double *gcexpo, int *KLMN);
/* replaces gpu_upload_cutoff_matrix_ (src/gpu/cuda/gpu.cu:879): YCutoff(nshell,nshell),
 * cutPrim(jbasis,jbasis) as computed by schwarzoff */
void gpu_upload_cutoff_matrix_(double *YCutoff, double *cutPrim);
/* replaces gpu_upload_calculated_ (src/gpu/cuda/gpu.cu:1690): density `dense` (nbasis^2) */
void gpu_upload_calculated_(double *o, double *co, double *vec, double *dense);
/* replaces gpu_upload_cutoff_ (src/gpu/cuda/gpu.cu:840): cutMatrix(nshell,nshell) and cutoffs */
void gpu_upload_cutoff_(double *cutMatrix, double *integralCutoff, double *primLimit,
                        double *DMCutoff, double *coreIntegralCutoff);
/* replaces gpu_get_cshell_eri_ (src/gpu/gpu_get2e_getxc_drivers.h:27, declared at
 * src/gpu/cuda/gpu.h:65): o(nbasis,nbasis) += G(dense), G = J - K/2 */
void gpu_get_cshell_eri_(bool *deltaO, double *o);
/* replaces gpu_upload_calculated_beta_ (src/gpu/cuda/gpu.cu, declared at src/gpu/cuda/gpu.h:33):
 * the beta density `denseb` (nbasis^2) of an open-shell (UHF) build */
void gpu_upload_calculated_beta_(double *ob, double *denseb);
/* replaces gpu_get_oshell_eri_ (src/gpu/gpu_get2e_getxc_drivers.h:24-25 under OSHELL):
 * o += G_alpha, ob += G_beta from the densities of gpu_upload_calculated_ (alpha) and
 * gpu_upload_calculated_beta_ (beta) and the open-shell density screen of gpu_upload_cutoff_ */
void gpu_get_oshell_eri_(bool *deltaO, double *o, double *ob);
/* replaces gpu_delete_ (src/gpu/cuda/gpu.cu:514) */
void gpu_delete_(int *ierr);

/* ======================================================= context API */
typedef struct qk_ctx qk_ctx;

/* Status of the most recent failing call (QK_OK if none since gpu_new_, which
 * starts a drop-in session). */
int qk_last_status(void);
const char *qk_status_string(int status);
/* Rows of gccoeff/gcexpo expected by gpu_upload_basis_ (reference MAXPRIM; default 20). */
int qk_set_maxprim(int maxprim);
/* Largest angular momentum per shell compiled into the kernels (3 = f). */
int qk_max_l(void);

/* Create / destroy a context on CUDA device `device`. */
qk_ctx *qk_create(int device, int *status);
int qk_destroy(qk_ctx *ctx);
/* The process-wide context the drop-in entry points use (created on first use). */
qk_ctx *qk_default_ctx(void);

/* Molecule + basis in QUICK layout (arguments as in gpu_upload_basis_, restricted to
 * what get2e needs).  xyz(3,natom) Bohr; kstart/katom/kprim/Ksumtype 1-based. */
int qk_set_basis(qk_ctx *ctx, int natom, const double *xyz, int nshell, int nbasis, int jbasis,
                 const int *kstart, const int *katom, const int *kprim, const int *Ksumtype,
                 const int *Qstart, const int *Qfinal, const int *Qsbasis, const int *Qfbasis,
                 const double *gccoeff, const double *cons, const double *gcexpo,
                 const int *KLMN, int maxprim);

/* Schwarz bounds on the GPU (replaces schwarzoff, src/modules/quick_cutoff_module.f90:54-89):
 * YCutoff(nshell,nshell) and cutPrim(jbasis,jbasis) written to host arrays (may be NULL)
 * and installed in the context. */
int qk_schwarz(qk_ctx *ctx, double *YCutoff, double *cutPrim);
/* Install caller-provided Schwarz bounds (same layout as gpu_upload_cutoff_matrix_). */
int qk_set_schwarz(qk_ctx *ctx, const double *YCutoff, const double *cutPrim);
/* integralCutoff and primLimit (src/modules/quick_method_module.f90:772-775).  Every
 * build applies the cutoffs in force (the CPU get2e's tests Y_ij*Y_kl > cut and
 * Y_ij*Y_kl*DNmax > cut).  The work lists are rebuilt only when the cutoff tightens
 * below the one they were built at: an SCF that tightens its cutoff as it converges
 * (adjust_Cutoff, src/modules/quick_method_module.f90:1107-1129) sets the final cutoff,
 * calls qk_prepare, then loosens it, and the lists are built once. */
int qk_set_cutoffs(qk_ctx *ctx, double integralCutoff, double primLimit);
/* Mixed precision (no counterpart in the reference, which is FP64 throughout): quartets
 * whose Schwarz bound product Y_ij*Y_kl is below fp32_bound evaluate the vertical
 * recursion and the primitive contraction in FP32; the Boys function, geometry, HRR,
 * digestion and the fixed-point accumulation stay FP64, as do the high angular
 * momentum (cooperative) classes.  0 (the default) = plain FP64. */
int qk_set_precision(qk_ctx *ctx, double fp32_bound);
/* Boys function of the integral kernels.  0 (the default): a 7-term Taylor step from a
 * tabulated grid below T = 36, the asymptotic form above, accurate to ~2e-15 relative for
 * every order used.  1 and 2: QUICK's own formulas (src/subs/fmt.f90:13-85; device copy
 * src/gpu/gpu_fmt.h:5-72) operation by operation, to reproduce the reference's Fock
 * matrices -- including their first-order branch below T = 0.1 and the precision their
 * upward recursion loses for high orders at small T.  Mode 1 evaluates at the order
 * QUICK's CPU get2e uses (the shell quartet's, SP shells counting 1: eri.fh:259, 394);
 * mode 2 at the order of the split s/p class, as QUICK's GPU get2e does
 * (src/gpu/gpu_get2e_subs.h:266).  Applies to the Fock builds and to qk_schwarz. */
int qk_set_boys(qk_ctx *ctx, int mode);
/* Shell quartets of the current work lists that run in FP32 (mixed form). */
int qk_last_work_mixed(qk_ctx *ctx, long long *quartets_fp32);

/* o_dev += G(D_dev).  D_dev, o_dev: nbasis^2 FP64 on the device.  cutmat_dev: nshell^2
 * density screen (max |D| per shell pair) or NULL to derive it from D_dev on the device
 * (cshell_density_cutoff, src/modules/include/cutoff.fh:62-92).  Enqueued on `stream`
 * (a cudaStream_t; NULL = the CUDA default stream); returns without synchronising.
 * The first call after a basis or Schwarz change, or after the cutoff tightens below
 * the one the lists were built at, also builds the pair tables and work lists on the
 * host and waits for their upload. */
int qk_fock2e_device(qk_ctx *ctx, const double *D_dev, const double *cutmat_dev,
                     double *o_dev, void *stream);
/* Same with host buffers: D and o are copied to the device, G is added into o there
 * and o is copied back; synchronises.  Pinned host buffers make the copies fastest. */
int qk_fock2e_host(qk_ctx *ctx, const double *D, const double *cutmat, double *o);
/* Density screen on the device: cutmat_dev(nshell,nshell) = max |D| per shell pair
 * (stream: a cudaStream_t, NULL = the CUDA default stream). */
int qk_density_cutoff_device(qk_ctx *ctx, const double *D_dev, double *cutmat_dev, void *stream);

/* Open-shell (UHF) Fock build (replaces get_oshell_eri, src/modules/include/eri.fh under
 * OSHELL, and its GPU form src/gpu/gpu_get2e_subs.h:638-660): oa_dev += G_alpha,
 * ob_dev += G_beta with G_alpha = J[Da + Db] - K[Da] and G_beta = J[Da + Db] - K[Db]
 * (HF exchange).  cutmat_dev: QUICK's open-shell density screen (per shell pair the
 * largest of |Da + Db|, |Da|, |Db|; oshell_density_cutoff, src/modules/include/cutoff.fh)
 * or NULL to derive it on the device.  Computed as a closed-shell build of Da + Db and an
 * exchange-only build of Da - Db on the same screened quartets; bit-reproducible.
 * Enqueued on `stream`, no synchronisation; the _host form copies and synchronises. */
int qk_fock2e_uhf_device(qk_ctx *ctx, const double *Da_dev, const double *Db_dev, const double *cutmat_dev,
                         double *oa_dev, double *ob_dev, void *stream);
int qk_fock2e_uhf_host(qk_ctx *ctx, const double *Da, const double *Db, const double *cutmat, double *oa,
                       double *ob);

/* Allocation-free Fock build (no counterpart in the reference).  Same arguments and
 * result as qk_fock2e_device, for callers that must not allocate device memory at the
 * point of the build -- a program that fixes its memory pool at start-up, or code
 * that may not call cudaMalloc/cudaFree because they synchronise the device.  The
 * per-build scratch (the fixed-point accumulator, the work counters and, when
 * cutmat_dev is NULL, the density screen) lives in one array inside the library that
 * every GPU loading it holds until exit: limits nbasis <= 1024 and, with
 * cutmat_dev == NULL, nshell <= 512; larger sizes return QK_ERR_INVALID_ARG.
 * The pair tables must already exist: run qk_fock2e_device (or qk_prepare) once after
 * any basis or Schwarz change, a tightening of the cutoff or a change of the FP32 bound
 * (qk_set_precision), else QK_ERR_NOT_READY.  The launch shape follows qk_set_streams,
 * and qk_last_work reports this build's counts.  The first call on a device looks
 * up the array's device address; make it before any stream capture.  All calls share
 * the array, so calls that overlap on the GPU race: keep them on one stream (or order
 * them with events). */
int qk_fock2e_device_noalloc(qk_ctx *ctx, const double *D_dev, const double *cutmat_dev,
                             double *o_dev, void *stream);

/* Sharded builds (the GPU form of the reference's MPI split of the work by cost,
 * MPI_setup_hfoperator, src/mpi_setup.f90:295-354, which deals bra shells to ranks greedily).
 * qk_set_shard: this context keeps every count-th work item (rank, rank + count, ...)
 * of each class's cost-ordered list; (0, 1) = all of them (the default).  The work
 * lists are rebuilt at the next build.  While count > 1 the finalising builds
 * (qk_fock2e_device, qk_fock2e_host, qk_fock2e_device_noalloc, qk_batch_fock2e) refuse
 * the context with QK_ERR_INVALID_ARG: they would return only this shard's part of G.
 * qk_fock2e_device_accumulate: the context's share of the build of G(D_dev) added
 * into A_dev, the caller's int64 fixed-point accumulator (nbasis^2 on the device,
 * 2^-44 units, cleared by the caller); nothing is finalised.  Summing the ranks'
 * accumulators (an integer all-reduce, exact and order-free) and calling
 * qk_finalize_fixed once gives, bit for bit, the unsharded build.
 * qk_finalize_fixed: o_dev(n,n) += (A + A^T) * 2^-44 on `stream`. */
int qk_set_shard(qk_ctx *ctx, int rank, int count);
int qk_fock2e_device_accumulate(qk_ctx *ctx, const double *D_dev, const double *cutmat_dev, long long *A_dev,
                                void *stream);
int qk_finalize_fixed(const long long *A_dev, int n, double *o_dev, void *stream);

/* Build the shell-pair tables and work lists for the current basis, Schwarz bounds,
 * cutoffs and precision now (the first Fock build does it otherwise), e.g. while
 * other work keeps the GPU busy.  Uses only the context's own stream. */
int qk_prepare(qk_ctx *ctx);

/* Device memory held by a context (pair tables, work lists, accumulators), in bytes;
 * *items = the part taken by the work lists (a batch holds one more copy of them). */
int qk_device_bytes(qk_ctx *ctx, unsigned long long *total, unsigned long long *items);

/* ------------------------------------------------------------- batches
 * Many molecules in one Fock build (no counterpart in the reference, which builds one
 * molecule per process): for every class one merged work list over all molecules,
 * launched once, so that small molecules fill the GPU together.  Each context keeps
 * its own tables, cutoffs and precision; o_dev[m] += G(D_dev[m]) for every molecule.
 * cutmat_dev may be NULL (or hold NULL entries) to screen from D on the device.  The
 * merged lists are cached and rebuilt when the set of contexts or their lists change. */
typedef struct qk_batch qk_batch;
qk_batch *qk_batch_create(int device, int *status);
int qk_batch_destroy(qk_batch *batch);
int qk_batch_fock2e(qk_batch *batch, int n, qk_ctx *const *ctx, const double *const *D_dev,
                    const double *const *cutmat_dev, double *const *o_dev, void *stream);
/* Size the batch's persistent class kernels for all SMs but `sms` (default 0), so
 * that other work on the GPU -- e.g. the set-up of new molecules on other streams
 * -- finds free SMs while a batch runs.  Same results. */
int qk_batch_reserve_sms(qk_batch *batch, int sms);

/* Work statistics of the last build: shell quartets listed and primitive quartets
 * listed after Schwarz screening (before density screening), and the kernel
 * launches that build made (before any build: those the next build will make). */
int qk_last_work(qk_ctx *ctx, long long *quartets, long long *prim_quartets, int *launches);
/* Kernel launches of one build (for launch accounting). */
int qk_launches_per_build(qk_ctx *ctx);

/* Who builds the work lists (the quartet items each class kernel walks): 1 (the
 * default) the GPU -- one thread per (bra pair, ket bucket) finds its Schwarz-admitted
 * ket prefix, scans place the items, two small host synchronisations; 0 the host (the
 * reference implementation of the lists, also used by sharded contexts).  Both give
 * the same lists item for item.  The reference builds its pair list on the host
 * (gpu_upload_cutoff_matrix_, src/gpu/cuda/gpu.cu:879-1470). */
int qk_set_worklist_builder(qk_ctx *ctx, int on_device);

/* The six per-lane s/p classes (ssss, psss, psps, ppss, ppps, pppp) as one
 * persistent kernel per precision over their joined work lists, heaviest class
 * first (on = 1), instead of one launch per class (0, the default).  The Fock
 * matrix is the same bit for bit; the merged kernel runs every class at the
 * register allocation of the largest.  The reference walks all classes in one
 * kernel over the pair-list product (src/gpu/gpu_get2e_subs.h:771).  Applies to
 * qk_fock2e_device and the calls built on it, not to the allocation-free build,
 * the many-molecule batch or builds with per-class profiling on. */
int qk_set_merge_sp(qk_ctx *ctx, int on);

/* A stream of the caller's own: non-blocking, at the device's highest priority
 * (high_priority != 0) or its lowest, owned by nobody else.  Streams handed out by a
 * framework's pool may be shared with other threads; a thread that captures a CUDA
 * graph needs one that no other thread can enqueue work on.  Free it with
 * qk_stream_destroy once its work is done.  No reference counterpart (QUICK runs one
 * SCF per process on the default stream). */
int qk_stream_create(int device, int high_priority, void **stream);
int qk_stream_destroy(void *stream);

/* Launch shape of a build: the class kernels run concurrently over `nstreams`
 * auxiliary streams forked from the caller's stream (1..4, default 4), or one after
 * another on the caller's stream (0).  A tuning knob: which is faster depends on
 * the molecule's mix of classes. */
int qk_set_streams(qk_ctx *ctx, int nstreams);

/* Launch shape of one integral class (index as listed by qk_class_profile):
 * warps per block (1..max, 0 = default: 4 for the per-lane classes, the
 * shared-memory fit for the cooperative ones) and a cap on resident blocks per SM
 * (0 = as many as fit).  The grid stays persistent (blocks loop over the class's
 * work items), so any shape computes the same result.  qk_class_launch reads the
 * shape in force, the largest allowed warps per block and the current grid. */
int qk_set_class_launch(qk_ctx *ctx, int cls, int warps_per_block, int blocks_per_sm);
int qk_class_launch(qk_ctx *ctx, int cls, int *warps_per_block, int *max_warps, int *blocks_per_sm, int *grid);

/* Per-class measurement: `events` records CUDA events around every class launch on the
 * launching stream; `stats` counts the quartets and primitive quartets each class
 * actually evaluated (after density and primitive screening). */
int qk_set_profiling(qk_ctx *ctx, int events, int stats);
/* Per-class figures of the last build: cls[4*i] = (La, Lb, Lc, Ld), kernel time in ms,
 * quartets / primitive quartets listed and evaluated, and the algorithmic FP64
 * operations per primitive quartet and per quartet.  Returns the number of classes,
 * or a negative status. */
int qk_class_profile(qk_ctx *ctx, int max_classes, int *cls, float *ms, long long *q_listed,
                     long long *pq_listed, long long *q_done, long long *pq_done,
                     double *prim_flops, double *quartet_flops);
/* FP64 FMA throughput of device `device` measured by a short probe kernel (GFLOP/s). */
int qk_fp64_peak(int device, double *gflops);
/* Diagnostic: the Boys function F_0..F_M (M <= 4 * qk_max_l()) at n points T[i] >= 0
 * (host arrays), evaluated on the device by the two forms the Fock kernels use: the
 * per-lane kernels' evaluation of all orders at once (F_rows) and the cooperative
 * kernels' one-order evaluation (F_one), in the context's qk_set_boys mode;
 * out[i*(M+1) + m].  No counterpart in the reference, whose device Boys is
 * src/gpu/gpu_fmt.h:5-72.  Synchronises. */
int qk_boys(qk_ctx *ctx, int M, const double *T, int n, double *F_rows, double *F_one);

/* Solve the n x n system A x = b (row-major device arrays, n <= 64) on `stream`
 * with partial pivoting, in one warp; *ok_dev = 1, or 0 (and x = 0) when a pivot
 * vanishes.  The DIIS step of an SCF iteration that stays on the device (no host
 * synchronisation, so the iteration can be captured in a CUDA graph); QUICK
 * solves the same system on the host (src/modules/quick_scf_module.f90:165-802). */
int qk_small_solve(const double *A_dev, const double *b_dev, int n, double *x_dev, int *ok_dev, void *stream);
/* One SP2 purification step on `stream` (no counterpart in the reference, which
 * diagonalises): given Y and Y2 = Y Y (n x n device arrays), Yout = Y2 when
 * |tr Y2 - nocc| < |2 tr Y - tr Y2 - nocc|, else 2Y - Y2 (Niklasson, Phys. Rev. B 66,
 * 155115 (2002)).  Yout must not alias Y or Y2.  The traces and the update are one
 * launch, so a captured SCF iteration holds two nodes per step (the GEMM and this). */
int qk_sp2_step(const double *Y_dev, const double *Y2_dev, double *Yout_dev, int n, double nocc, void *stream);
/* `steps` SP2 steps on `stream`, each the GEMM Y2 = Y Y (cuBLAS DGEMM) and
 * qk_sp2_step, with Ya and Yb as ping-pong buffers: the purified matrix ends in Ya
 * when `steps` is even, in Yb when it is odd.  One call instead of 2 x steps, so that
 * a host loop -- or the capture of one into a CUDA graph -- costs one call whatever
 * the step count.  The first call on a device creates the library's cuBLAS handle
 * for that device (steps = 0 does only that): it must come before any stream
 * capture; inside a capture it returns QK_ERR_NOT_READY instead.  The handle runs
 * without a workspace, so calls on different streams share no scratch memory. */
int qk_sp2_run(double *Ya_dev, double *Yb_dev, double *Y2_dev, int n, double nocc, int steps, void *stream);

/* One-electron integrals on device `device` (replaces the get1e path and the
 * reference's gpu_get_oei_, src/gpu/gpu_oei.cu:194; CPU twin
 * src/modules/quick_oei_module.f90:69-257).  Basis in QUICK's normalize_basis
 * layout: ncontract(nbasis), itype(3,nbasis), aexp/dcoeff(maxcontract,nbasis),
 * ncenter(nbasis) 1-based.  Charges: nuclei Z(natom) at xyz(3,natom) plus `next`
 * external point charges ext_q at ext_xyz(3,next) (QM/MM).  Writes S, T, V
 * (nbasis^2, symmetric) to host arrays; functions up to f. */
int qk_oei_host(int device, int natom, const double *xyz, const double *Z, int nbasis,
                int maxcontract, const int *ncontract, const int *itype, const double *aexp,
                const double *dcoeff, const int *ncenter, int next, const double *ext_xyz,
                const double *ext_q, double *S, double *T, double *V);

#ifdef __cplusplus
}
#endif

#endif /* QUICK_B200_H */
