// Host-side launchers of the FP64 kernels.  Internal to the library (the public
// C-ABI is include/zolo_b200.h).  All matrices are column-major FP64 in device
// memory; every launcher takes an explicit stream and returns cudaError_t.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace zolo {

// C(b) = alpha * a_b * op(A(b)) * op(B(b)) + beta * C(b),  b = 0..batch-1
struct GemmArgs {
  int M = 0, N = 0, K = 0;
  int transA = 0, transB = 0;
  const double* A = nullptr;
  int64_t lda = 0, strideA = 0;
  const double* B = nullptr;
  int64_t ldb = 0, strideB = 0;
  double* C = nullptr;
  int64_t ldc = 0, strideC = 0;
  double alpha = 1.0, beta = 0.0;
  const double* alpha_vec = nullptr;  // per-batch factor a_b (device), nullptr = 1
  int batch = 1;
  int tri = 0;      // 1: M == N, write only C(i,j) with i >= j (lower triangle)
  int kfrom_n = 0;  // 1: op(B)(k,n) == 0 for k < n (op(B) lower triangular): skip those k;
                    // 2: op(A)(m,k) == 0 for k < m (op(A) upper triangular): skip those k;
                    // 3: both (k from max(row, column))
  int kto_m = 0;    // 1: op(A)(m,k) == 0 for k > m (op(A) lower triangular): skip those k;
                    // 2: op(B)(k,n) == 0 for k > n (op(B) upper triangular): skip those k
  int splitk = 0;   // 0 = choose; 1 = off; >1 = number of K slices
};

// Scratch for split-K partial sums (owned by the caller's context).
struct Scratch {
  double* ptr = nullptr;
  size_t bytes = 0;
};

cudaError_t dgemm(GemmArgs a, const Scratch& ws, cudaStream_t st);
size_t dgemm_splitk_bytes(const GemmArgs& a, int num_sms);
// Streaming rank-k update C = beta*C + alpha*A*B (no transposes, K <= 32; update.cu).
// dgemm dispatches to it when rank_update_applies(a).
bool rank_update_applies(const GemmArgs& a);
cudaError_t rank_update(const GemmArgs& a, cudaStream_t st);

// ---- FP64 products emulated on the INT8 tensor cores (ozaki.cu) ----
// C = alpha op(A) op(B) + beta C (batched, tri / kfrom_n / kto_m as in GemmArgs; no
// alpha_vec) from S = `slices` (6..8) signed 7-bit digit planes of each operand, products
// accumulated exactly in INT32 (requires slices * 127^2 * K < 2^31, ozgemm_k_ok).
// Workspace sizes from ozgemm_work_bytes.  Device status codes 901..906: a pipeline wait
// timed out.
struct OzWorkSizes {
  size_t slice_a = 0, slice_b = 0;  // bytes of digit planes
  size_t rows_a = 0, rows_b = 0;    // padded rows (one max and one exponent per row)
};
struct OzWork {
  int8_t* sliceA = nullptr;
  int8_t* sliceB = nullptr;
  unsigned long long* maxA = nullptr;
  unsigned long long* maxB = nullptr;
  int* expA = nullptr;
  int* expB = nullptr;
  int* status = nullptr;
  // optional: recorded on the stream right before the INT8 kernel's launch (after the
  // splitting), so that a caller can time the splitting and the kernel apart
  cudaEvent_t before_kernel = nullptr, before_kernel2 = nullptr;
};
size_t ozgemm_work_bytes(const GemmArgs& a, int slices, OzWorkSizes* sz);
bool ozgemm_k_ok(int slices, int K);
cudaError_t ozgemm(const GemmArgs& a, int slices, const OzWork& w, cudaStream_t st, int sms);

// ---- elementwise / reductions (elementwise.cu) ----
// dst(i,j) = s * src(i,j) (+ d on the diagonal), batched.
cudaError_t scale_copy(int m, int n, double s, const double* src, int64_t lds, int64_t strideS,
                       double* dst, int64_t ldd, int64_t strideD, int batch, double diag_add,
                       cudaStream_t st);
// W = [X; 0; s I]: X (m x n) in rows [0,m), zeros in [m,mpad), s I in rows [mpad, mpad+n)
// (mpad >= m keeps the identity block at an even row offset), batched over s_vec[b] or s_scalar.
// x_upper: take only the upper triangle of X (zeros below its diagonal).  strideX: X of
// batch entry b at X + b*strideX (0: one X shared by the batch, the r Zolotarev terms).
cudaError_t form_stack(int m, int mpad, int n, const double* X, int64_t ldx, double* W, int64_t ldw,
                       int64_t strideW, const double* s_vec, double s_scalar, int batch,
                       cudaStream_t st, int x_upper = 0, int64_t strideX = 0);
// dst(b) = lower(G) + c_b I (lower triangle + diagonal only), batched.
cudaError_t shift_lower(int n, const double* G, int64_t ldg, double* W, int64_t ldw,
                        int64_t strideW, const double* c_vec, int batch, cudaStream_t st);
// Sum of squares partials -> out[0] = ||X||_F^2 (deterministic two-pass).
cudaError_t frob2(int m, int n, const double* X, int64_t ldx, double* partial, double* out,
                  cudaStream_t st);
// out[0] = max_j sum_i |X(i,j)|
cudaError_t norm1(int m, int n, const double* X, int64_t ldx, double* colsum, double* out,
                  cudaStream_t st);
// X <- cx X + sum_q w_q Z_q, w_q = cz_vec[q] (device) or cz; err2 = ||X_new - X_old||_F^2
// (FormX2 of Zolo-PD with w_q = a_q / FONE, cx = 1/FONE; QDWH update with cx = bkk, cz = akk)
cudaError_t combine_update(int m, int n, double* X, int64_t ldx, const double* Z, int64_t ldz,
                           int64_t strideZ, int nz, double cx, double cz, const double* cz_vec,
                           double* partial, double* err2, cudaStream_t st);
// H = (B + B^T)/2 (in place on an n x n matrix).
cudaError_t symmetrize(int n, double* B, int64_t ldb, cudaStream_t st);
// B = scale * triu(A) (n x n; zero below the diagonal)
cudaError_t copy_upper(int n, const double* A, int64_t lda, double scale, double* B, int64_t ldb, cudaStream_t st);
// B = A^T
cudaError_t transpose(int m, int n, const double* A, int64_t lda, double* B, int64_t ldb,
                      cudaStream_t st);
// Q = [I; 0] (m x n, batched)
// Newton-Schulz step matrix: with `write`, G (lower triangle of X^T X on entry) <-
// (3I - G)/2, both triangles; always *err2 = ||G_in - I||_F^2 (partial: >= 1024
// doubles of scratch).
cudaError_t ns_prepare(int n, double* G, int64_t ldg, double* partial, double* err2, int write, cudaStream_t st);
// B's upper triangle = its lower triangle mirrored (B n x n)
cudaError_t mirror_lower(int n, double* B, int64_t ldb, cudaStream_t st);
cudaError_t set_identity(int m, int n, double* Q, int64_t ldq, int64_t strideQ, int batch,
                         double diag, cudaStream_t st);
// A(i,i) += d
cudaError_t add_diag(int n, double* A, int64_t lda, double d, cudaStream_t st);
// sum of a device vector of partials into out (helper used by reductions)
cudaError_t reduce_sum(const double* partial, int count, double* out, cudaStream_t st);

// ---- Cholesky / triangular (potrf.cu) ----
// In-place lower Cholesky of nb x nb blocks (nb <= 64), batched; LAPACK INFO (+info_offset)
// recorded in info[b]; when Dinv != nullptr the inverse of the factor goes to
// Dinv + b*strideD (64 x 64, ld 64, zeros above the diagonal).
cudaError_t potrf_leaf(int nb, double* A, int64_t lda, int64_t strideA, int batch, int* info,
                       int info_offset, double* Dinv, int64_t strideD, cudaStream_t st);
// Inverses of all 64 x 64 diagonal blocks of lower-triangular n x n matrices:
// block kb of batch entry b -> Dinv + (b*nblk + kb)*4096, nblk = ceil(n/64).
cudaError_t trtri_blocks(int n, const double* L, int64_t ldl, int64_t strideL, double* Dinv, int batch,
                         cudaStream_t st);

// ---- Householder QR panel (qr.cu) ----
// Factor the m x w panel of each batch entry (w <= 32) in place: V below the
// diagonal (unit diagonal implied), R on/above it, tau[w], T (w x w upper, ld 32)
// of the compact WY form I - V T V^T.  Vexp receives V explicitly (m x w, ldv).
// Row gap: with split > 0, logical row r >= split of the panel is the physical
// row r + gap of A (two row segments; Vexp stays in logical rows).
cudaError_t qr_panel(int m, int w, double* A, int64_t lda, int64_t strideA, double* tau,
                     int64_t strideTau, double* T, int64_t strideT, double* Vexp, int64_t ldv,
                     int64_t strideV, int batch, cudaStream_t st, int split = 0, int64_t gap = 0);
// Cluster size the panel kernel uses for an m x w panel (negative: rows stay in global memory).
int qr_panel_config(int m, int w);
// Vexp = unit-lower-trapezoidal V taken from A (m x w logical rows, same row gap
// as qr_panel), batched.
cudaError_t extract_v(int m, int w, const double* A, int64_t lda, int64_t strideA, double* V,
                      int64_t ldv, int64_t strideV, int batch, cudaStream_t st, int split = 0,
                      int64_t gap = 0);
// TB(b) (jb x jb, ld ldtb) <- block diagonal of the ceil(jb/32) consecutive 32 x 32 panel T
// factors at T + b*strideT (ld 32, 1024 apart), zero elsewhere.
cudaError_t block_t_init(int jb, const double* T, int64_t strideT, double* TB, int64_t ldtb, int64_t strideTB,
                         int batch, cudaStream_t st);
// P'(b) = T(b)^T * P(b) (trans=1) or T(b) * P(b) (trans=0); T w x w upper (ld 32), P w x n.
cudaError_t apply_t(int w, int n, const double* T, int64_t strideT, double* P, int64_t ldp,
                    int64_t strideP, int trans, int batch, cudaStream_t st);

// ---- eigen stage (jacobi.cu, elementwise.cu) ----
struct JacobiLeaf {
  const double* A;  // n x n symmetric (read)
  int64_t lda;
  int n;            // <= 64
  double* w;        // eigenvalues (unsorted)
  double* V;        // eigenvectors (n x n, ldv)
  int64_t ldv;
};
// One CTA per leaf (device array of descriptors); sweeps[i] receives the sweep count.
cudaError_t jacobi_leaves(const JacobiLeaf* d_leaves, int count, int max_sweeps, int* d_sweeps, cudaStream_t st);
// X(i,j) = uniform(-1,1) from a counter hash of (seed, i, j)
cudaError_t fill_random(int m, int n, double* X, int64_t ldx, uint64_t seed, cudaStream_t st);
// out[0] = sum_i A(i,i)
cudaError_t trace(int n, const double* A, int64_t lda, double* out, cudaStream_t st);
// B(:, j) = A(:, perm[j])
cudaError_t gather_columns(int m, int n, const double* A, int64_t lda, const int* perm, double* B, int64_t ldb,
                           cudaStream_t st);
// d[i] = A(i,i)
cudaError_t get_diag(int n, const double* A, int64_t lda, double* d, cudaStream_t st);

int num_sms();

// ---- batched polar decomposition (batch.cu) ----
// One matrix of a batch: A (m x n) in, Q (m x n) and H (n x n, may be null) out, and
// the value tau of the identity block that pads it to the bucket size.
struct BatchMember {
  int m, n;
  const double* A;
  int64_t lda;
  double tau;
  double* Q;
  int64_t ldq;
  double* H;
  int64_t ldh;
};
// P(b) = [[A_b, 0], [0, tau_b I], [0, 0]] (MB x NB)
cudaError_t batch_pack(const BatchMember* d_mem, int count, int MB, int NB, double* P, int64_t ldp, int64_t sp,
                       cudaStream_t st);
// Q_b = Q'(b)[0:m, 0:n], H_b = H'(b)[0:n, 0:n]
cudaError_t batch_unpack(const BatchMember* d_mem, int count, int MB, int NB, const double* Q, int64_t ldq,
                         int64_t sq, const double* H, int64_t ldh, int64_t sh, cudaStream_t st);
// out[b] = ||X_b||_F^2 (partial: partial_cap doubles of scratch)
cudaError_t batch_frob2(int m, int n, const double* X, int64_t ldx, int64_t sx, int batch, double* partial,
                        int partial_cap, double* out, cudaStream_t st);
// out[b] = ||X_b||_1 (largest column sum of absolute values)
cudaError_t batch_norm1(int m, int n, const double* X, int64_t ldx, int64_t sx, int batch, double* out,
                        cudaStream_t st);
// X_b <- s[b] X_b
cudaError_t batch_scale(int m, int n, double* X, int64_t ldx, int64_t sx, int batch, const double* s,
                        cudaStream_t st);
// X_b <- cx[b] X_b + cz[b] Z_b (cz[b] = 0 leaves X_b as it is), err2[b] = ||X_b,new - X_b||_F^2
cudaError_t batch_combine(int m, int n, double* X, int64_t ldx, int64_t sx, const double* Z, int64_t ldz, int64_t sz,
                          int batch, const double* cx, const double* cz, double* partial, int partial_cap,
                          double* err2, cudaStream_t st);
// Conditional steps of the batched solver's schedule: where cond[b] != 0 and
// sqrt(err2_prev[b]) <= tol, member b's coefficients in `row` (coef, cx, cz; batch entries
// each) become neutral for the step's form (qr: 1, 1, 0; Cholesky: 0, 1, 0).
cudaError_t batch_gate(int batch, const double* err2_prev, const double* cond, double* row, int qr, double tol,
                       cudaStream_t st);
cudaError_t batch_add_diag(int n, double* G, int64_t ldg, int64_t sg, int batch, double d, cudaStream_t st);
cudaError_t batch_symmetrize(int n, double* B, int64_t ldb, int64_t sb, int batch, cudaStream_t st);
cudaError_t batch_transpose(int m, int n, const double* A, int64_t lda, int64_t sa, double* B, int64_t ldb,
                            int64_t sb, int batch, cudaStream_t st);

}  // namespace zolo
