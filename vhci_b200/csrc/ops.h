// Host launchers for the device kernels.  All launches are asynchronous on the given stream.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"

namespace vhci {

// Process-wide count of this library's kernel launches (reported in vhci_stats).
void note_launch();
long long launch_count();

// ---- device table records ----
struct GroupDev {   // one connection group (a fixed quanta change)
  int32_t tb, te;   // term range
  uint8_t nchg;
  uint8_t mode[6];
  int8_t delta[6];
  uint8_t pad[3];
};
struct TermDev {    // one FC term of a group: fc * prod_j T[pw_j][q(mode_j)][dl_j]
  double fc;
  uint8_t nk;
  uint8_t mode[6];
  uint8_t pw[6];
  int8_t dl[6];
  uint8_t pad[5];
};
struct HBDev {      // heat-bath list entry (pattern decoder)
  int32_t zero_idx;
  uint8_t nk;
  uint8_t mode[6];
  uint8_t pw[6];
  uint8_t pad[3];
};
static_assert(sizeof(GroupDev) == 24, "GroupDev layout");
static_assert(sizeof(TermDev) == 32, "TermDev layout");
static_assert(sizeof(HBDev) == 20, "HBDev layout");

struct ConnDev {            // connection tables on device
  const GroupDev* groups;
  const int64_t* wdelta;    // [ngroups * W] packed key change per word
  int64_t ngroups;
  const TermDev* terms;
  const TermDev* dterms;    // Delta = 0 terms
  int ndterms;
  const double* T;          // ladder table, (qmax+1) stride
  const double* freq;       // [nm]
  int nm;
  // lowered-mode index: open-addressing table of the group segments (groups are ordered by the
  // key of the modes they lower; see ConnTables)
  const uint64_t* lkey;     // [lmask + 1] segment keys, 0 = empty slot
  const int32_t* lseg;      // [2 (lmask + 1)] first group and group count of the segment
  uint32_t lmask;
  int maxl;                 // most modes one group lowers; -1: no index, visit every group
};

struct HBTable {
  const HBDev* e;
  const double* absfc;      // [nhb] |fc| descending
  const int64_t* cum;       // [nhb+1] exclusive prefix of pattern counts
  int nhb;
};

// ---- scan / utilities (k_basis.cu) ----
// Exclusive prefix sum of n int64 values into out (may alias in); returns nothing, total is
// written to out[n] (out must hold n+1).  tmp must hold scan_tmp_elems(n) int64.
int64_t scan_tmp_elems(int64_t n);
void exclusive_scan(const int64_t* in, int64_t* out, int64_t n, int64_t* tmp, cudaStream_t s);
void exclusive_scan_i32(const int32_t* in, int64_t* out, int64_t n, int64_t* tmp, cudaStream_t s);

// ---- keys and hash ----
void pack_keys(const uint8_t* quanta, int64_t n, int nm, KeyLayout L, uint64_t* keys,
               cudaStream_t s);
void unpack_keys(const uint64_t* keys, int64_t n, int nm, KeyLayout L, uint8_t* quanta,
                 cudaStream_t s);
void repack_keys(const uint64_t* in, KeyLayout from, uint64_t* out, KeyLayout to, int64_t n,
                 int nm, cudaStream_t s);
void hash_clear(uint64_t* slots, uint64_t nslots, cudaStream_t s);
void hash_insert_range(uint64_t* slots, uint64_t mask, const uint64_t* keys, int64_t begin,
                       int64_t end, int W, int* flags, cudaStream_t s);
void max_quanta_per_mode(const uint64_t* keys, int64_t n, int nm, KeyLayout L, int* out,
                         cudaStream_t s);

// ---- heat-bath selection ----
// cmax[i] = signed C_ij of max |C_ij| over j < nopt (first occurrence); X row-major, ld = ldx.
void cmax_rows(const double* X, int64_t n, int ldx, int nopt, double* cmax, cudaStream_t s);
// work[i] = number of patterns generated by state i at threshold eps.
void select_count(const double* cmax, int64_t n, HBTable hb, double eps, int64_t* work,
                  cudaStream_t s);
// Generate candidates for work items [0, total): probe the basis hash, insert absent keys into
// the new-state set.
void select_generate(const uint64_t* keys, int64_t n, const int64_t* woff, int64_t total,
                     HBTable hb, KeyLayout L, HashView basis, NewSetView ns, cudaStream_t s);
// Compact live candidates into out (count written to *n_out on device).
void newset_compact(const uint64_t* cand, const uint8_t* dead, int64_t ncand, int W,
                    uint64_t* out, unsigned long long* n_out, cudaStream_t s);

// ---- radix sort of packed keys (ascending, most significant word last) ----
// Sorts n keys of W words in place using `alt` (n*W words) as the ping-pong buffer; only the low
// `nbits` bits of the key (mode fields in use) are examined.  hist must hold
// radix_hist_elems(n) int64.
int64_t radix_hist_elems(int64_t n);
void radix_sort_keys(uint64_t* keys, uint64_t* alt, int64_t n, int W, int nbits, int64_t* hist,
                     cudaStream_t s);

// ---- Hamiltonian (k_ham.cu) ----
// Incremental build (the stored rows of the first n_old states plus the rows of the nn states
// appended since; H is symmetric to the bit).  hmerge_cross_keys: add[c] += 1 and a key
// (c << 32 | e) for every new-row entry e in an old column c (cnt[0] counts the keys, in no fixed
// order).  hmerge_entry_rows: erow[e] = the new row of entry e.  hmerge_lengths: merged row
// lengths.  hmerge_copy_rows: rows [rs[i], rs[i+1]) to offset rd[i] (FP64 values, or FP32 when
// vsf is given).  hmerge_cross_scatter: the sorted keys to the tails of the old rows (xoff:
// exclusive scan of add).
void hmerge_cross_keys(const int32_t* col_new, int64_t nnz_new, int64_t n_old, int32_t* add,
                       uint64_t* keys, unsigned long long* cnt, cudaStream_t s);
void hmerge_entry_rows(const int64_t* rp_new, int64_t nn, int32_t* erow, cudaStream_t s);
void hmerge_lengths(const int64_t* rp_old, const int32_t* add, const int64_t* rp_new, int64_t n_old,
                    int64_t nn, int32_t* len, cudaStream_t s);
void hmerge_copy_rows(const int64_t* rs, const int32_t* cs, const double* vs, const float* vsf,
                      int64_t nrows, const int64_t* rd, int32_t* cd, double* vd, float* vdf,
                      cudaStream_t s);
void hmerge_cross_scatter(const uint64_t* keys, int64_t ncross, const int64_t* xoff,
                          const int64_t* rp_old, const int64_t* rp_all, const int32_t* erow,
                          const double* vnew, const float* vnewf, int64_t n_old, int32_t* cd,
                          double* vd, float* vdf, cudaStream_t s);
// Rows row0 .. row0 + n - 1 of the Hamiltonian (rowcnt, rowptr, diag indexed from row0).
void hbuild_count(const uint64_t* keys, int64_t row0, int64_t n, KeyLayout L, HashView basis,
                  ConnDev cd, int32_t* rowcnt, cudaStream_t s);
void hbuild_fill(const uint64_t* keys, int64_t row0, int64_t n, KeyLayout L, HashView basis,
                 ConnDev cd, const int64_t* rowptr, int32_t* col, double* val, float* valf,
                 double* diag, cudaStream_t s);
// Column panels of the off-diagonal CSR (at most kMaxPanels): entries of panel p (columns
// [p cw, (p+1) cw)) for row i at [prow[p n + i], prow[p n + i + 1]).
constexpr int kMaxPanels = 64;
void panel_count(int64_t n, const int64_t* rowptr, const int32_t* col, int64_t cw, int32_t* cnt,
                 cudaStream_t s);
void panel_fill(int64_t n, const int64_t* rowptr, const int32_t* col, const double* val,
                const float* valf, int64_t cw, int P, const int64_t* prow, int32_t* pcol,
                double* pval, float* pvalf, cudaStream_t s);
// Y[:, 0:b] = H X[:, 0:b] for the n rows of a CSR (or column-panelled) matrix of FP64 or FP32
// off-diagonal values plus the FP64 diagonal; the diagonal term of row i multiplies X row
// xrow0 + i (0 unless the rows are one rank's block of a sharded matrix).
void spmm_panels(int64_t n, int P, const int64_t* prow, const int32_t* pcol, const double* pval,
                 const float* pvalf, const double* diag, const double* X, int ldx, int b,
                 double* Y, int ldy, int64_t xrow0, cudaStream_t s);
void spmm(int64_t n, const int64_t* rowptr, const int32_t* col, const double* val,
          const float* valf, const double* diag, const double* X, int ldx, int b, double* Y,
          int ldy, int64_t xrow0, cudaStream_t s);
// Mixed precision: FP32 values and FP32 gathered block X (16-byte aligned, b and ldx multiples of
// 4), FP64 accumulation; the diagonal term multiplies the FP64 block Xd (row i of the rows held).
// Returns false (nothing launched) when the shapes do not allow the 16-byte gathers.
bool spmm_f32x(int64_t n, const int64_t* rowptr, const int32_t* col, const float* val,
               const double* diag, const float* X, int ldx, int b, const double* Xd, int ldd,
               double* Y, int ldy, cudaStream_t s);
void copy_cols_f32(const double* src, int lds, float* dst, int ldd, int64_t n, int ncol,
                   cudaStream_t s);
// ---- eigensolver helpers ----
// rn2[c] (c < kk) = sum_i (HX[i,c] - theta[c] X[i,c])^2   (block partials reduced on device)
void residual_norms(const double* X, const double* HX, int64_t n, int ld, int kk,
                    const double* theta, double* part, int nblk, double* rn2, cudaStream_t s);
int residual_blocks(int64_t n);
void copy_cols(const double* src, int lds, double* dst, int ldd, int64_t n, int ncol,
               cudaStream_t s);
void dense_from_csr(int64_t n, const int64_t* rowptr, const int32_t* col, const double* val,
                    const float* valf, const double* diag, double* A, cudaStream_t s);
void fill_zero(double* p, int64_t n, cudaStream_t s);

// ---- FP64 tensor-core projections (k_proj.cu) ----
// C (M x P, column-major, ldc) = alpha A^T B + beta C with A n x M and B n x P row-major (lda,
// ldb); any M (slabs of 1024), P <= 16; part holds proj_gram_scratch(M, P) doubles.  Returns
// false (nothing launched) for P > 16 or strides shorter than the rows.
int64_t proj_gram_scratch(int M, int P);
bool proj_gram(const double* A, int lda, const double* B, int ldb, int64_t n, int M, int P,
               double alpha, double beta, double* C, int ldc, double* part, cudaStream_t s);
// Out (n x P row-major, ldo) = alpha A S + beta Out with A n x M row-major and S M x P
// column-major (lds); any P (column chunks of 64).
void proj_rows(const double* A, int lda, const double* S, int lds, int64_t n, int M, int P,
               double alpha, double beta, double* Out, int ldo, cudaStream_t s);
// W <- W - A S1, then C (M x P, column-major) = A^T W, in one pass over A; M <= 768, P <= 16
// (false, nothing launched, otherwise); part holds proj_gram_scratch(M, P) doubles.
bool proj_rows_gram(const double* A, int lda, const double* S1, int lds, double* W, int ldw,
                    int64_t n, int M, int P, double* C, int ldc, double* part, cudaStream_t s);
// SVQB factor M (nb x nb, column-major) of the Gram matrix S = W^T W (nb <= 16) on the device:
// W M is orthonormal over the directions above 1e-12 of the largest, further columns of M are
// zero and *rank_short is set to 1 when there are any.
void svqb_factor(const double* S, int nb, double* M, int* rank_short, cudaStream_t s);

// ---- PT2 (k_pt2.cu) ----
void pt2_count(const uint64_t* keys, int64_t n, KeyLayout L, HashView pert, ConnDev cd,
               int64_t a_lo, int64_t a_hi, int32_t* acount, cudaStream_t s);
void pt2_fill(const uint64_t* keys, int64_t n, KeyLayout L, HashView pert, ConnDev cd,
              int64_t a_lo, int64_t a_hi, const int64_t* arowptr, int32_t* afill, int32_t* ecol,
              double* eval, cudaStream_t s);
// Fused EN reduction over perturbers [a_lo, a_hi): num_a = sum_e eval_e X[ecol_e, :nopt];
// E_a = harmonic + diagonal terms; part[blk][n] += num^2 / (E_n - E_a).
// Every block writes all nopt columns of its part row; any nopt >= 1 (column tiles of 256);
// returns false for an unsupported key width or nopt < 1 (nothing launched).
int pt2_en_blocks();
bool pt2_en(const uint64_t* pkeys, int64_t a_lo, int64_t a_hi, KeyLayout L, ConnDev cd,
            const int64_t* arowptr, const int32_t* ecol, const double* eval, const double* X,
            int ldx, int nopt, const double* E, double* part, cudaStream_t s);
// Orders the entries of each perturber row [arowptr[r], arowptr[r+1]) by ascending state index,
// so the EN sums run in one fixed order.  pt2_sort_rows handles rows shorter than
// pt2_sort_long_min() entries; pt2_sort_long the listed longer rows (rows[q], with scratch
// tcol/tval of their total length, row q's part at soff[q]).
void pt2_sort_rows(const int64_t* arowptr, int64_t nrows, int32_t* ecol, double* eval,
                   cudaStream_t s);
int pt2_sort_long_min();
// crow[i] = arow[i] - arow[0] for i in [0, nrows]
void pt2_rebase_rows(const int64_t* arow, int64_t nrows, int64_t* crow, cudaStream_t s);
// rows of at least pt2_sort_long_min() entries into rows[] with disjoint scratch offsets soff[]
// (cnt[0] += rows listed, cnt[1] += their entries; both zeroed by the caller)
void pt2_list_long(const int64_t* arowptr, int64_t nrows, int64_t* rows, int64_t* soff,
                   unsigned long long* cnt, cudaStream_t s);
void pt2_sort_long(const int64_t* arowptr, const int64_t* rows, const int64_t* soff, int nlong,
                   int32_t* ecol, double* eval, int32_t* tcol, double* tval, cudaStream_t s);
void reduce_parts(const double* part, int nblk, int nopt, double* out_accum, cudaStream_t s);

}  // namespace vhci
