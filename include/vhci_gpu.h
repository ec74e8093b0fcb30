/*
 * vhci_gpu.h — C ABI of the B200 (sm_100a) heat-bath VCI + Epstein-Nesbet PT2 library.
 *
 * The reference program (berkelbach-group/VHCI) is one C++ binary with global state and no plugin
 * or FFI layer.  This ABI exposes, as plain C calls over host pointers and sizes, the internal
 * seams of that program; each declaration names the reference function it stands in for.  The
 * `vhci` command-line tool (drop-in for `vhci -n/-i/-o/-c`) and the Python harness (ctypes) are
 * both written on top of it.
 *
 * Conventions
 *  - Every call returns a vhci_status (0 = OK).  vhci_last_error() gives the message.
 *  - The caller owns every host buffer; the context owns all device memory and one CUDA stream.
 *  - A context is used by one host thread at a time; separate contexts may run concurrently.
 *  - There is no CPU fallback: without a usable CUDA device, vhci_create* returns VHCI_E_CUDA.
 *  - Basis states are passed as rows of per-mode quanta, uint8_t[n * nmodes], row-major.
 *  - Eigenvectors are passed column-major, double[n * k] (column j = state j), as the reference's
 *    Eigen MatrixXd.
 */
#ifndef VHCI_GPU_H
#define VHCI_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int vhci_status;
enum {
  VHCI_OK = 0,
  VHCI_E_INPUT = 1,         /* malformed input file / arguments (reference: message + exit)     */
  VHCI_E_OOM = 2,           /* device memory exhausted                                           */
  VHCI_E_TABLE_FULL = 3,    /* a device hash table could not take a key within its probe bound   */
  VHCI_E_KEY_OVERFLOW = 4,  /* a state needs more than 255 quanta in one mode                    */
  VHCI_E_NOT_CONVERGED = 5, /* eigensolver hit its iteration limit (reference: Ham.cpp:367-368)  */
  VHCI_E_CUDA = 6,          /* CUDA runtime / library failure                                    */
  VHCI_E_STATE = 7,         /* call made in the wrong state (e.g. no vectors yet)                */
  VHCI_E_NEG_ZPE = 8,       /* zero-point energy < 0 (reference: VHCI.cpp:122-137)               */
  VHCI_E_LIMIT = 9          /* the basis or perturber space would exceed max_basis / max_pert    */
};

typedef struct vhci_ctx vhci_ctx;

/* Options.  Fill with vhci_default_opts() and change fields as needed. */
typedef struct {
  int device;          /* CUDA device ordinal                                                   */
  int precision;       /* 0: FP64 throughout (parity path); 1: mixed — FP32 Hamiltonian values
                          with FP64 accumulation, FP64 Ritz steps, PT2 denominators and a final
                          FP64 residual sweep                                                    */
  double eig_tol;      /* relative residual tolerance, reference 1e-10 (Ham.cpp:363)            */
  int eig_maxit;       /* eigensolver iteration bound, reference 1000 (Ham.cpp:363)             */
  int verbose;         /* 1: print the reference's progress lines to stdout                    */
  int host_threads;    /* host threads for host-side steps (reference -n)                       */
  int64_t pt2_chunk;   /* max perturber-Hamiltonian entries held at once (0 = automatic)        */
  int structural_nnz;  /* 1: the verbose "% sparse" line uses the reference's structural count
                          (vhci_structural_nnz; one extra counting pass per build), falling
                          back to the stored entries when that count is unavailable           */
  int64_t max_basis;   /* 0 = no limit; else a heat-bath iteration whose selection would grow the
                          basis past this fails with VHCI_E_LIMIT before building H             */
  int64_t max_pert;    /* 0 = no limit; else PT2 fails with VHCI_E_LIMIT when the screened
                          perturber space is larger, before the perturber Hamiltonian is built  */
  int stream_priority; /* priority of the context's CUDA stream (cudaStreamCreateWithPriority:
                          lower numbers run first, clamped to the device's range; 0 = default)  */
} vhci_opts;

/* Problem description in memory (the content of a reference input file, Input_Reader.cpp). */
typedef struct {
  int nmodes;               /* Nm                                                              */
  const double* freq;       /* [nmodes] harmonic frequencies (cm^-1)                           */
  const int* cap;           /* [nmodes] per-mode quanta cap of the initial basis               */
  int max_quanta;           /* Ntot: initial basis = all states with sum of quanta <= Ntot     */
  int nfc;                  /* number of anharmonic force constants                            */
  const int* fc_order;      /* [nfc] order 3..6                                                */
  const int* fc_modes;      /* [nfc * 6] mode indices (first fc_order[i] used)                 */
  const double* fc_value;   /* [nfc] unscaled values as written in the input file              */
  double eps1;              /* HCI_Eps (0 = conventional VCI over the initial basis)           */
  int nstate;               /* Nstate                                                          */
  int pt2;                  /* PT2 flag                                                        */
  double eps2;              /* PT2_Eps (0 = every connected state)                             */
} vhci_problem;

typedef struct {
  int nmodes, nstate, pt2, key_bits, key_words;
  double eps1, eps2;
  int64_t n_basis;          /* current variational basis size                                  */
  int64_t n_fc, n_hb;       /* scaled FCs; heat-bath list (FCs + aggregated singles/doubles)   */
  int64_t n_groups;         /* distinct quanta-change patterns of the FC list (H connections)  */
  int64_t n_vectors;        /* eigenpairs currently held                                       */
  int64_t h_nnz;            /* stored off-diagonal Hamiltonian entries (0 if not built)        */
} vhci_info;

/* Per-phase device time of the most recent solve (milliseconds) and work counters. */
typedef struct {
  double ms_select, ms_hbuild, ms_eigs, ms_pt2, ms_total;
  double ms_spmm;                 /* part of ms_eigs spent in the SpMM kernel                  */
  int64_t spmm_calls, spmm_cols;  /* SpMM launches and total vector columns multiplied         */
  int64_t spmm_bytes;             /* algorithmic bytes of all SpMM launches                    */
  int64_t hbuild_probes;          /* hash probes issued by the Hamiltonian build               */
  int64_t select_candidates;      /* candidate states generated by heat-bath selection         */
  int64_t pt2_entries;            /* perturber-Hamiltonian entries (a, i, H_ai)                */
  int64_t pt2_perturbers;         /* |P|                                                       */
  double ms_pt2_reduce;           /* part of ms_pt2 spent in the fused EN reduction kernel     */
  int64_t pt2_reduce_bytes;       /* algorithmic bytes of the EN reduction                     */
  int eig_iterations;             /* Davidson iterations summed over all eigensolves           */
  int hci_iterations;
  int64_t h2d_bytes, d2h_bytes;   /* host<->device bytes copied by the library                 */
  int64_t kernel_launches;        /* this library's kernel launches so far (process-wide)      */
  int64_t spmm_gather_bytes;      /* vector-row bytes the sparse products gathered (nnz * b * 8
                                     per product, 4 with FP32 gathers): the traffic that bounds
                                     them, mostly from L2                                       */
  double mixed_max_residual;      /* mixed precision: largest ||H x - theta x|| / max(1, |theta|)
                                     of the Ritz pairs after the FP64 sweeps                     */
  int64_t hbuild_incremental;     /* Hamiltonian builds that extended the stored matrix by the
                                     rows of the newly added states (no counterpart in the
                                     reference, which rebuilds H every heat-bath iteration)      */
} vhci_stats;

typedef void (*vhci_iter_cb)(void* user, int iteration, int64_t n_basis, double zpe);

void vhci_default_opts(vhci_opts* o);

/* Parse an input file with the reference's positional rules (Input_Reader.cpp:170-291), scale
 * the FCs (ScaleFC, :494-515), build the heat-bath list (:366-460, HB.cpp:17-22) and the initial
 * basis (:295-364), and upload everything.  restart != 0 starts from the ground state only, as
 * the reference does before reading a checkpoint (:296-307). */
vhci_status vhci_create_from_file(const char* path, const vhci_opts* o, int restart,
                                  vhci_ctx** out);
/* Same from an in-memory problem. */
vhci_status vhci_create(const vhci_problem* p, const vhci_opts* o, int restart, vhci_ctx** out);
vhci_status vhci_destroy(vhci_ctx* c);
vhci_status vhci_last_error(const vhci_ctx* c, char* buf, size_t n);
vhci_status vhci_get_info(const vhci_ctx* c, vhci_info* info);
vhci_status vhci_get_stats(const vhci_ctx* c, vhci_stats* s);
vhci_status vhci_reset_stats(vhci_ctx* c);

/* Scaled FC list in input order and the sorted heat-bath list: value plus up to 6 (mode, power)
 * pairs (mode -1 pads).  Parity dumps of Input_Reader.cpp:249-291,366-460 and HB.cpp:17-22. */
vhci_status vhci_get_fc_list(const vhci_ctx* c, double* value, int32_t* modes, int32_t* powers);
vhci_status vhci_get_hb_list(const vhci_ctx* c, double* value, int32_t* modes, int32_t* powers);
/* Harmonic frequencies as parsed. */
vhci_status vhci_get_freqs(const vhci_ctx* c, double* freq);

/* Basis I/O (the reference's BasisSet).  set_basis replaces the basis and drops vectors. */
vhci_status vhci_set_basis(vhci_ctx* c, const uint8_t* quanta, int64_t n);
vhci_status vhci_get_basis(const vhci_ctx* c, uint8_t* quanta, int64_t cap, int64_t* n);

/* Eigenpairs (the reference's Evecs/Evals).  set_vectors injects caller vectors (n x k,
 * column-major) for selection/PT2 known-answer tests; get_vectors copies k of them out. */
vhci_status vhci_set_vectors(vhci_ctx* c, const double* C, const double* E, int k);
vhci_status vhci_get_vectors(const vhci_ctx* c, double* C, double* E, int k);

/* Heat-bath selection, AddStatesHB over all states (HB.cpp:24-174, driver :198-223) with
 * Cmax over the first min(nstate, n) vector columns.  append != 0 appends the new states (in
 * ascending key order) and updates the device hash; otherwise they are kept for
 * vhci_get_selected().  n_new receives the number of new states. */
vhci_status vhci_select(vhci_ctx* c, double eps, int append, int64_t* n_new);
vhci_status vhci_get_selected(const vhci_ctx* c, uint8_t* quanta, int64_t cap, int64_t* n);

/* Sparse Hamiltonian over the current basis (MakeHamSparse, Ham.cpp:203-344), kept on device.
 * nnz receives the stored entry count including the diagonal. */
vhci_status vhci_build_h(vhci_ctx* c, int64_t* nnz);
/* Copy the Hamiltonian out as CSR with columns ascending in every row (nnz from build_h). */
vhci_status vhci_get_h_csr(const vhci_ctx* c, int64_t* rowptr, int32_t* col, double* val);
/* Entry count of the reference's stored Hamiltonian pattern (Ham.cpp:236-344): the diagonal plus
 * every ordered pair of basis states whose quanta pass its gates, structural zeros included; the
 * "% sparse" line prints 100 (1 - count / N^2) (Ham.cpp:341-342).  Works on the current basis
 * (no Hamiltonian needed); VHCI_E_LIMIT when the gates admit more than 2,000,000 change patterns
 * (many modes with 6th-order terms). */
vhci_status vhci_structural_nnz(vhci_ctx* c, int64_t* nnz);

/* Y = H X for b host vectors (n x b, column-major) with the current Hamiltonian (built on first
 * use): the sparse product the eigensolver runs (SparseSymMatProd in the reference, Ham.cpp:349). */
vhci_status vhci_apply_h(vhci_ctx* c, const double* X, double* Y, int b);

/* Residual norms || H x_j - theta_j x_j || of k host vectors (n x k, column-major) with the
 * current Hamiltonian: the convergence measure of the reference's eigensolver (Ham.cpp:363). */
vhci_status vhci_residual_norms(vhci_ctx* c, const double* X, const double* theta, double* rnorm,
                                int k);
/* The same residual norms for callers that cannot allocate device memory when they need them (a
 * serving process whose device memory belongs to its own pool, or code that must avoid the implicit
 * device-wide synchronisation of cudaMalloc/cudaFree).  No counterpart in the reference.
 * Inputs and outputs are DEVICE pointers on the context's device: X_dev is n x k row-major
 * (ld = k), theta_dev has k values, rnorm_dev receives k values; results are ready when the call
 * returns.  The call allocates nothing: its scratch is a fixed array of 296 x 256 doubles (606 KB)
 * in the library's device memory, which every device that loads the library keeps until the
 * process exits.  Limits and rules:
 *  - 1 <= k <= 256, else VHCI_E_INPUT;
 *  - the Hamiltonian must already be built (vhci_build_h), else VHCI_E_STATE;
 *  - X_dev, theta_dev and rnorm_dev must be device memory of the context's device (checked with
 *    cudaPointerGetAttributes, else VHCI_E_INPUT);
 *  - the work runs on the context's own stream, which does not wait for the caller's streams:
 *    the inputs must be complete when the call is made (e.g. synchronise the stream that wrote
 *    them first);
 *  - the caller's current device is left as it was;
 *  - the first call on a device looks up the scratch array's device address (and may load the
 *    library's device code); make that first call before any stream capture.  The address is
 *    kept for the life of the process: after a cudaDeviceReset of that device neither it nor any
 *    context created before the reset may be used;
 *  - all calls share the one array: calls whose work overlaps on the GPU (from several threads or
 *    contexts on one device) race and must be serialised by the caller. */
vhci_status vhci_residual_norms_noalloc(vhci_ctx* c, const double* X_dev, const double* theta_dev,
                                        double* rnorm_dev, int k);

/* Lowest k eigenpairs of the current Hamiltonian (SparseDiagonalize, Ham.cpp:347-370; dense
 * eigensolve for small bases, DenseDiagonalize, :372-379).  Vectors stay on device; E (k)
 * receives the eigenvalues if not NULL. */
vhci_status vhci_eigs(vhci_ctx* c, int k, double* E);

/* Full heat-bath procedure (Perform_HCI, HB.cpp:176-265) or, for eps1 == 0, one eigensolve over
 * the initial basis (VHCI.cpp:49-76).  checkpoint_path may be NULL; when given, a checkpoint is
 * written after each iteration whose basis exceeds 1e5 states (HB.cpp:250-262). */
vhci_status vhci_hci(vhci_ctx* c, const char* checkpoint_path, vhci_iter_cb cb, void* user);

/* Epstein-Nesbet PT2 (DoPT2, PT2.cpp:16-154) over the current vectors.  dE (min(nstate, n))
 * receives the corrections, which are also added to the held eigenvalues.  n_pert receives |P|. */
vhci_status vhci_pt2(vhci_ctx* c, double eps2, double* dE, int64_t* n_pert);

/* Frequency/assignment file (PrintFreqs, Ham.cpp:448-502). */
vhci_status vhci_write_freqs(const vhci_ctx* c, const char* path);
/* Checkpoint text file (WriteCheckpoint / ReadCheckpoint, Core_functions.cpp:94-167). */
vhci_status vhci_write_checkpoint(const vhci_ctx* c, const char* path);
vhci_status vhci_read_checkpoint(vhci_ctx* c, const char* path);

/* Eigenvalues currently held (n <= k). */
vhci_status vhci_get_energies(const vhci_ctx* c, double* E, int k, int* n);

/* ---- one solve sharded over several GPUs ---------------------------------------------------
 * No counterpart in the reference program, which runs in one address space (its loops are OpenMP
 * threads over one basis, Ham.cpp:237, PT2.cpp:66).  With a communicator set, the ranks (one
 * context per GPU, each built from the same input) solve one problem together:
 *  - the Hamiltonian's rows and the eigensolver's Krylov basis are split into contiguous row
 *    blocks of ceil(n / nranks) rows, one per rank;
 *  - before every sparse product the ranks' blocks of the vector block are all-gathered, and the
 *    projections' partial sums (Gram matrices, residual norms) are all-reduced; the projected
 *    eigenproblem is solved on rank 0 and broadcast;
 *  - after each eigensolve the Ritz vectors are all-gathered, so heat-bath selection runs on every
 *    rank with identical results;
 *  - PT2 splits the perturber space into one contiguous range per rank and all-reduces the
 *    corrections.
 * The collectives are the caller's (for example torch.distributed over NCCL).  The library
 * synchronises its stream before each call; a callback must finish the collective (the buffers
 * are device memory of the context's device) before it returns 0.  Every rank must make the same
 * sequence of library calls.  Bases whose eigensolve is dense (up to 2000 states, and the first
 * heat-bath step) are solved whole on every rank.  vhci_apply_h, vhci_residual_norms(_noalloc)
 * and vhci_get_h_csr return VHCI_E_STATE on a sharded context. */
typedef struct {
  int rank, nranks;
  void* user;
  /* sum `count` doubles of buf over the ranks, in place */
  int (*allreduce_sum)(void* user, double* buf, int64_t count);
  /* recv (nranks * bytes bytes) = the ranks' `bytes`-byte send buffers in rank order */
  int (*allgather)(void* user, const void* send, void* recv, int64_t bytes);
} vhci_comm;

/* Set (or, with NULL or nranks == 1, clear) the communicator; call before vhci_hci. */
vhci_status vhci_set_comm(vhci_ctx* c, const vhci_comm* comm);

/* ---- request server (continuous batching of independent solves on one GPU) ----------------
 * No counterpart in the reference program, which solves one input per process.  Each request is
 * a reference-format input file (or an in-memory problem) with an arrival time in seconds after
 * the call starts.  A request is admitted into one of `slots` workers once it has arrived, a slot
 * is free and the device's free memory is at least `reserve_bytes` (or nothing else runs); every
 * admitted request has its own context and CUDA stream, so concurrent requests overlap on the GPU.
 * A request that runs out of device memory is retried after another request finishes.
 * Energies of request i go to energies[i * max_states ...] (first n_energies values). */
typedef struct {
  const char* input_path;          /* input file, or NULL to use `problem`                      */
  const vhci_problem* problem;
  double arrival_s;                /* arrival time after the start of vhci_serve                */
} vhci_request;

typedef struct {
  int device;
  int slots;                       /* concurrent requests (default 8)                           */
  double reserve_bytes;            /* free device memory required to admit (default 8e9)        */
  int max_states;                  /* energies stored per request (default 256)                 */
  int64_t max_basis, max_pert;     /* per-request size limits, as in vhci_opts (default 0: none)  */
  int fifo_priority;               /* 1 (default): a request admitted while others run gets a lower
                                      stream priority than all of them, so the earliest requests
                                      finish about as fast as alone and later ones fill the gaps  */
} vhci_serve_opts;

typedef struct {
  int status;                      /* vhci_status of the request                                */
  int worker, retries, n_energies;
  int64_t n_basis, n_pert;
  double t_admit, t_done;          /* seconds after the start of vhci_serve                     */
  char message[160];
} vhci_result;

typedef struct {
  double wall_s;
  int completed, failed, peak_in_flight;
} vhci_serve_summary;

void vhci_default_serve_opts(vhci_serve_opts* so);
vhci_status vhci_serve(const vhci_request* reqs, int nreq, const vhci_serve_opts* so,
                       vhci_result* results, double* energies, vhci_serve_summary* summary);

#ifdef __cplusplus
}
#endif
#endif /* VHCI_GPU_H */
