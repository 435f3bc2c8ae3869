// Leaf Cholesky factorisation fused with the inversion of the factor, for one
// diagonal block of at most 64 columns: a device function run by one CTA of
// 256 threads, shared by the blocked factorisation's leaf kernel and the
// persistent tile-task kernel of batched small instances.
#ifndef MOAO_LEAF_F64_CUH
#define MOAO_LEAF_F64_CUH

namespace moao {

constexpr int LEAF = 64;
constexpr int LEAF_LD = LEAF + 1;
constexpr int LEAF_TRI = LEAF * (LEAF + 1) / 2;  // 2,080
// shared memory of leaf_factor_inverse, bytes
constexpr int LEAF_SMEM_BYTES = (2 * LEAF * LEAF_LD + 3 * LEAF) * 8;

// Leaf factorisation of a diagonal block (n <= 64) fused with the inversion of
// its triangular factor, one CTA of THREADS threads (all of which call it).
// Every thread owns up to OWN = ceil(2,080 / THREADS) elements of the 64 x 64
// lower triangle (element e = t + THREADS s of the row-packed triangle) and
// keeps them in registers through both phases:
//   factor (right-looking, step j = 0..63): the owners of column j publish it
//     (unscaled) to shared memory, and the owner of A(j,j) publishes
//     r = 1/sqrt(A(j,j)); after one barrier every thread writes
//     L(i,j) = A(i,j) r (L(j,j) = A(j,j) r) for its column-j elements and
//     applies A(i,k) -= (A(i,j) r)(A(k,j) r) to its elements with k > j
//     (column j is never written during step j);
//   inverse (X = L^-1 by rows, step i = 0..63, B = I): the owners of row i
//     finish X(i,c) = B(i,c) / L(i,i) and publish the row; after one barrier
//     every thread applies B(r,c) -= L(r,i) X(i,c) to its elements with r > i.
// The published column/row alternates between two buffers, so one barrier per
// step suffices: a thread can only overwrite a buffer after every thread has
// passed the next step's barrier, i.e. finished reading it. A non-positive
// pivot is reported (first failing global column, 1-based, into *info) and
// replaced by 1 so the kernel finishes without NaNs; rows and columns beyond n
// are an identity block. Only the n x n parts of A (lower) and Linv are
// written. A is read through L2 (ld.global.cg): in the tile-task kernel other
// SMs wrote it moments before.

template <int THREADS>
__device__ __forceinline__ void leaf_factor_inverse(double* A, long lda, double* Linv, long ldi,
                                                    int n, long col0, int* info,
                                                    double* leaf_smem) {
  constexpr int LEAF_THREADS = THREADS;
  constexpr int LEAF_OWN = (LEAF_TRI + THREADS - 1) / THREADS;
  double* Lf = leaf_smem;                     // the factor, column-major, ld LEAF_LD
  double* Xs = leaf_smem + LEAF * LEAF_LD;    // the input block, then the inverse
  double* buf = leaf_smem + 2 * LEAF * LEAF_LD;  // [2][LEAF]: published column / row
  double* rinv = buf + 2 * LEAF;              // 1 / L(j,j)
  const int tid = threadIdx.x;
  for (int e = tid; e < LEAF * LEAF; e += LEAF_THREADS) {
    const int i = e % LEAF, j = e / LEAF;
    Xs[i + j * LEAF_LD] = (i < n && j < n) ? (i >= j ? __ldcg(A + (long)j * lda + i) : 0.0)
                                           : (i == j ? 1.0 : 0.0);
  }
  __syncthreads();
  double a[LEAF_OWN];
  int ri[LEAF_OWN], ci[LEAF_OWN];  // row >= column of each owned element; -1 past the triangle
#pragma unroll
  for (int s = 0; s < LEAF_OWN; ++s) {
    const int e = tid + LEAF_THREADS * s;
    if (e < LEAF_TRI) {
      int i = (int)((sqrtf(8.0f * (float)e + 1.0f) - 1.0f) * 0.5f);  // row of the packed index
      while (i * (i + 1) / 2 > e) --i;
      while ((i + 1) * (i + 2) / 2 <= e) ++i;
      ri[s] = i;
      ci[s] = e - i * (i + 1) / 2;
      a[s] = Xs[ri[s] + ci[s] * LEAF_LD];
    } else {
      ri[s] = ci[s] = -1;
      a[s] = 0.0;
    }
  }
  // ---- factor
  for (int j = 0; j < LEAF; ++j) {
    double* cj = buf + (j & 1) * LEAF;
#pragma unroll
    for (int s = 0; s < LEAF_OWN; ++s) {
      if (ci[s] == j) {
        if (ri[s] == j) {  // the pivot: checked, its reciprocal square root published
          if (!(a[s] > 0.0)) {
            if (j < n) atomicCAS(info, 0, (int)(col0 + j + 1));
            a[s] = 1.0;
          }
          rinv[j] = rsqrt(a[s]);
        }
        cj[ri[s]] = a[s];
      }
    }
    __syncthreads();
    const double r = rinv[j];
#pragma unroll
    for (int s = 0; s < LEAF_OWN; ++s) {
      if (ci[s] == j) {
        Lf[ri[s] + j * LEAF_LD] = a[s] * r;
      } else if (ci[s] > j) {
        const double li = cj[ri[s]] * r, lk = cj[ci[s]] * r;
        a[s] = fma(-li, lk, a[s]);
      }
    }
  }
  __syncthreads();
  // ---- inverse of the factor, by rows
#pragma unroll
  for (int s = 0; s < LEAF_OWN; ++s) a[s] = (ri[s] >= 0 && ri[s] == ci[s]) ? 1.0 : 0.0;
  for (int i = 0; i < LEAF; ++i) {
    double* xi = buf + (i & 1) * LEAF;
    const double ri_inv = rinv[i];
#pragma unroll
    for (int s = 0; s < LEAF_OWN; ++s)
      if (ri[s] == i) {
        a[s] *= ri_inv;
        xi[ci[s]] = a[s];
      }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < LEAF_OWN; ++s)
      if (ri[s] > i && ci[s] <= i) a[s] = fma(-Lf[ri[s] + i * LEAF_LD], xi[ci[s]], a[s]);
  }
#pragma unroll
  for (int s = 0; s < LEAF_OWN; ++s)
    if (ri[s] >= 0) Xs[ri[s] + ci[s] * LEAF_LD] = a[s];
  __syncthreads();
  for (int e = tid; e < n * n; e += LEAF_THREADS) {
    const int i = e % n, j = e / n;
    if (i >= j) A[(long)j * lda + i] = Lf[i + j * LEAF_LD];
    Linv[(long)j * ldi + i] = i >= j ? Xs[i + j * LEAF_LD] : 0.0;
  }
}

}  // namespace moao

#endif  // MOAO_LEAF_F64_CUH
