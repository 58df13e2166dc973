/*
 * CPU oracle: a plain-C restatement of the reference VBCSR algorithms on the
 * hot path.  TEST INFRASTRUCTURE ONLY -- tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg use it as the checker; the shipped library never
 * links or loads it.  It is pinned against the reference itself
 * (oracle/_ref/libvbcsr_ref.so, built from the reference sources by
 * oracle/build_ref.sh) and against golden vectors under tests/golden/.
 *
 * Matrices are serial CSR-of-blocks: n block rows, block_sizes[n], row_ptr[n+1],
 * col_ind[nnzb] (sorted per row), values in slot order with row-major blocks
 * (vbcsr/core/block_csr.hpp:1202-1248 get_values).  Complex values are
 * interleaved (re, im).  Multivectors are dense row-major N x k.
 *
 * Floating-point order: the sums that feed integer/structure decisions (block
 * Frobenius norms, the SpGEMM symbolic norm-product sums) are evaluated in the
 * reference source's order without contraction (compiled with
 * -ffp-contract=off), which reproduces the reference binary's norms bit for
 * bit on all but ~0.1% of blocks; the remainder differ in the last ulp where
 * the reference's compiler fused an update into an FMA.  Decisions taken on
 * sums within 1e-10 relative of the threshold are therefore not pinned.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int n;
  const int* bsz;
  const int* row_ptr;
  const int* col_ind;
  const double* vals; /* real: nnz doubles; complex: 2*nnz doubles */
  int is_complex;
} orc_mat;

static int64_t* slot_offsets(const orc_mat* A) {
  const int64_t nnzb = A->row_ptr[A->n];
  int64_t* off = (int64_t*)malloc(sizeof(int64_t) * (nnzb + 1));
  off[0] = 0;
  for (int i = 0; i < A->n; ++i)
    for (int s = A->row_ptr[i]; s < A->row_ptr[i + 1]; ++s)
      off[s + 1] = off[s] + (int64_t)A->bsz[i] * A->bsz[A->col_ind[s]];
  return off;
}

static int64_t* scalar_offsets(int n, const int* bsz) {
  int64_t* so = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
  so[0] = 0;
  for (int i = 0; i < n; ++i) so[i + 1] = so[i] + bsz[i];
  return so;
}

/* ------------------------------------------------------------------ apply */
/* Y = A X or Y = A^H X (dense row-major N x k).  Follows the row-direct
 * apply of vbcsr/core/detail/kernels/vbcsr_apply.hpp:193-244 / :277-340
 * (per row: zero the output rows, then accumulate every slot's block
 * product) and the adjoint scatter of :342-424. */
void orc_apply(const orc_mat* A, int k, const double* X, double* Y, int adjoint) {
  const int cw = A->is_complex ? 2 : 1;
  int64_t* off = slot_offsets(A);
  int64_t* so = scalar_offsets(A->n, A->bsz);
  const int64_t N = so[A->n];
  memset(Y, 0, sizeof(double) * N * k * cw);
  for (int i = 0; i < A->n; ++i) {
    const int r = A->bsz[i];
    for (int s = A->row_ptr[i]; s < A->row_ptr[i + 1]; ++s) {
      const int j = A->col_ind[s];
      const int c = A->bsz[j];
      const double* b = A->vals + off[s] * cw;
      for (int t = 0; t < r; ++t)
        for (int q = 0; q < c; ++q) {
          const int64_t e = (int64_t)t * c + q;
          /* forward: Y[i,t] += a * X[j,q]; adjoint: Y[j,q] += conj(a) * X[i,t] */
          const int64_t yr = adjoint ? so[j] + q : so[i] + t;
          const int64_t xr = adjoint ? so[i] + t : so[j] + q;
          for (int v = 0; v < k; ++v) {
            if (cw == 1) {
              Y[yr * k + v] = fma(b[e], X[xr * k + v], Y[yr * k + v]);
            } else {
              const double ar = b[2 * e], ai = adjoint ? -b[2 * e + 1] : b[2 * e + 1];
              const double xr_ = X[2 * (xr * k + v)], xi_ = X[2 * (xr * k + v) + 1];
              Y[2 * (yr * k + v)] += ar * xr_ - ai * xi_;
              Y[2 * (yr * k + v) + 1] += ar * xi_ + ai * xr_;
            }
          }
        }
    }
  }
  free(off);
  free(so);
}

/* Block Frobenius norms, sum of squares in element order
 * (vbcsr/core/block_csr.hpp:2487-2502). */
void orc_block_norms(const orc_mat* A, double* out) {
  int64_t* off = slot_offsets(A);
  const int64_t nnzb = A->row_ptr[A->n];
  for (int64_t s = 0; s < nnzb; ++s) {
    double sum = 0.0;
    for (int64_t e = off[s]; e < off[s + 1]; ++e) {
      if (A->is_complex) {
        const double re = A->vals[2 * e], im = A->vals[2 * e + 1];
        sum += fma(re, re, im * im);
      } else {
        sum += A->vals[e] * A->vals[e];
      }
    }
    out[s] = sqrt(sum);
  }
  free(off);
}

/* ------------------------------------------------------------------ KPM */
/* Unnormalised moments mu_n = sum_r <v0_r | T_n(A) | v0_r> of a real
 * symmetric A.
 *   two_moment = 0: the three-term recurrence of
 *     examples/ex08_graphene_dos.py:99-114 (one moment per product)
 *   two_moment = 1: examples/inp_nanocrystal_dos/kpm.py:40-74
 *     (mu_2n = 2<t_n,t_n> - mu_0, mu_2n+1 = 2<t_n+1,t_n> - mu_1) */
static double dot_all(const double* a, const double* b, int64_t n) {
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

void orc_kpm_moments(const orc_mat* A, int R, const double* V0, int M, int two_moment, double* mu) {
  int64_t* so = scalar_offsets(A->n, A->bsz);
  const int64_t len = so[A->n] * R;
  free(so);
  double* t0 = (double*)malloc(sizeof(double) * len);
  double* t1 = (double*)malloc(sizeof(double) * len);
  double* t2 = (double*)malloc(sizeof(double) * len);
  memcpy(t0, V0, sizeof(double) * len);
  mu[0] = dot_all(t0, t0, len);
  if (M >= 2) {
    orc_apply(A, R, t0, t1, 0);
    mu[1] = dot_all(V0, t1, len);
    if (two_moment && M > 2) mu[2] = 2.0 * dot_all(t1, t1, len) - mu[0];
    int n = 1;
    for (;;) {
      if (two_moment) {
        if (2 * n + 1 >= M) break;
      } else {
        if (n + 1 >= M) break;
      }
      orc_apply(A, R, t1, t2, 0);
      for (int64_t i = 0; i < len; ++i) t2[i] = 2.0 * t2[i] - t0[i];
      if (two_moment) {
        mu[2 * n + 1] = 2.0 * dot_all(t1, t2, len) - mu[1];
        if (2 * n + 2 < M) mu[2 * n + 2] = 2.0 * dot_all(t2, t2, len) - mu[0];
      } else {
        mu[n + 1] = dot_all(V0, t2, len);
      }
      double* tmp = t0;
      t0 = t1;
      t1 = t2;
      t2 = tmp;
      ++n;
    }
  }
  free(t0);
  free(t1);
  free(t2);
}

/* psi_out = sum_n c_n T_n(A) psi for complex A and a single vector
 * (examples/ex09_graphene_dynamics.py:102-133; vbcsr/utils.py:71-126 with
 * center 0, scale 1).  coeffs interleaved complex. */
void orc_cheb_apply(const orc_mat* A, int M, const double* coeffs, const double* psi, double* out) {
  int64_t* so = scalar_offsets(A->n, A->bsz);
  const int64_t N = so[A->n];
  free(so);
  double* v0 = (double*)malloc(sizeof(double) * 2 * N);
  double* v1 = (double*)malloc(sizeof(double) * 2 * N);
  double* v2 = (double*)malloc(sizeof(double) * 2 * N);
  memcpy(v0, psi, sizeof(double) * 2 * N);
  for (int64_t i = 0; i < N; ++i) {
    out[2 * i] = v0[2 * i] * coeffs[0] - v0[2 * i + 1] * coeffs[1];
    out[2 * i + 1] = v0[2 * i] * coeffs[1] + v0[2 * i + 1] * coeffs[0];
  }
  if (M > 1) {
    orc_apply(A, 1, v0, v1, 0);
    for (int64_t i = 0; i < N; ++i) {
      out[2 * i] += v1[2 * i] * coeffs[2] - v1[2 * i + 1] * coeffs[3];
      out[2 * i + 1] += v1[2 * i] * coeffs[3] + v1[2 * i + 1] * coeffs[2];
    }
  }
  for (int k = 2; k < M; ++k) {
    orc_apply(A, 1, v1, v2, 0);
    const double cr = coeffs[2 * k], ci = coeffs[2 * k + 1];
    for (int64_t i = 0; i < N; ++i) {
      v2[2 * i] = 2.0 * v2[2 * i] - v0[2 * i];
      v2[2 * i + 1] = 2.0 * v2[2 * i + 1] - v0[2 * i + 1];
      out[2 * i] += v2[2 * i] * cr - v2[2 * i + 1] * ci;
      out[2 * i + 1] += v2[2 * i] * ci + v2[2 * i + 1] * cr;
    }
    double* t = v0;
    v0 = v1;
    v1 = v2;
    v2 = t;
  }
  free(v0);
  free(v1);
  free(v2);
}

/* ------------------------------------------------------- random vectors */
/* Counter-based entries of vbcsr/core/random_vectors.hpp:52-160 (splitmix64,
 * Steele, Lea & Flood 2014) as used by DistMultiVector::set_random
 * (vbcsr/core/dist_multivector.hpp:335-373): Rademacher for real, random
 * phase for complex, normalised by 1/sqrt(N). */
static uint64_t sm64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}
static uint64_t ent_hash(uint64_t seed, uint64_t b, uint64_t r, uint64_t c) {
  uint64_t h = sm64(seed + 0x9e3779b97f4a7c15ULL);
  h = sm64(h ^ (b * 0xbf58476d1ce4e5b9ULL));
  h = sm64(h ^ (r * 0x94d049bb133111ebULL));
  return sm64(h ^ (c * 0xd6e8feb86659fd93ULL));
}

void orc_set_random(int n, const int* bsz, int k, uint64_t seed, int normalize, int is_complex, double* out) {
  int64_t* so = scalar_offsets(n, bsz);
  const double scale = normalize ? 1.0 / sqrt((double)so[n]) : 1.0;
  for (int b = 0; b < n; ++b)
    for (int t = 0; t < bsz[b]; ++t)
      for (int c = 0; c < k; ++c) {
        const uint64_t h = ent_hash(seed, (uint64_t)b, (uint64_t)t, (uint64_t)c);
        const int64_t e = (so[b] + t) * k + c;
        if (is_complex) {
          const double u = (double)(h >> 11) * (1.0 / 9007199254740992.0);
          const double th = 2.0 * M_PI * u;
          out[2 * e] = cos(th) * scale;
          out[2 * e + 1] = sin(th) * scale;
        } else {
          out[e] = ((h >> 63) ? 1.0 : -1.0) * scale;
        }
      }
  free(so);
}

/* --------------------------------------------------------------- SpGEMM */
typedef struct {
  int n;
  int* row_ptr;
  int* col_ind;
  double* vals;
  int64_t nnzb, nnz;
  int64_t stats[4]; /* symbolic blocks, final blocks, block products, flops */
} orc_result;

void orc_result_free(orc_result* r) {
  free(r->row_ptr);
  free(r->col_ind);
  free(r->vals);
  memset(r, 0, sizeof(*r));
}

static int cmp_int(const void* a, const void* b) {
  const int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

/* Frobenius filter (keep norm >= thr when thr > 0) applied in place to a
 * result, vbcsr/core/block_csr.hpp:1399-1528. */
static void filter_result(orc_result* C, const int* bsz, int is_complex, double thr) {
  if (thr <= 0.0) return;
  const int cw = is_complex ? 2 : 1;
  orc_mat view = {C->n, bsz, C->row_ptr, C->col_ind, C->vals, is_complex};
  double* norms = (double*)malloc(sizeof(double) * (C->nnzb + 1));
  orc_block_norms(&view, norms);
  int64_t* off = slot_offsets(&view);
  int* rp = (int*)malloc(sizeof(int) * (C->n + 1));
  int* ci = (int*)malloc(sizeof(int) * (C->nnzb + 1));
  double* v = (double*)malloc(sizeof(double) * (C->nnz * cw + 1));
  int64_t nb = 0, nv = 0;
  rp[0] = 0;
  for (int i = 0; i < C->n; ++i) {
    for (int s = C->row_ptr[i]; s < C->row_ptr[i + 1]; ++s) {
      if (norms[s] >= thr) {
        ci[nb++] = C->col_ind[s];
        const int64_t len = (off[s + 1] - off[s]) * cw;
        memcpy(v + nv, C->vals + off[s] * cw, sizeof(double) * len);
        nv += len;
      }
    }
    rp[i + 1] = (int)nb;
  }
  free(norms);
  free(off);
  free(C->row_ptr);
  free(C->col_ind);
  free(C->vals);
  C->row_ptr = rp;
  C->col_ind = ci;
  C->vals = v;
  C->nnzb = nb;
  C->nnz = nv / cw;
}

/* C = A B with threshold, following VBCSRSpMMExecutor::run
 * (vbcsr/core/detail/ops/spmm/vbcsr.hpp:70-115):
 *  symbolic  ops/spmm/common.hpp:508-735 -- per row, accumulate
 *            sum_k |A_ik| |B_kj| per column j in (A slot, B slot) order and
 *            keep j iff the sum > threshold; columns sorted (:664, :668)
 *  numeric   ops/spmm/vbcsr.hpp:206-471 -- per A slot (i,k), per B slot
 *            (k,j): skip when |A_ik||B_kj| < threshold / max(1, nnzblk(A row))
 *            (:372, :386), skip when j is not in C's row, else
 *            C_ij += A_ik B_kj
 *  filter    C.filter_blocks(threshold) (block_csr.hpp:1399-1528).
 * upper != 0: only block columns j >= i (symbolic_multiply_filtered's
 * upper_only, common.hpp:502-506, :625); the numeric phase follows the
 * pattern, so it computes the upper triangle only. */
static void spgemm_impl(const orc_mat* A, const orc_mat* B, double thr, int upper, orc_result* C) {
  const int n = A->n;
  const int cw = A->is_complex ? 2 : 1;
  double* nA = (double*)malloc(sizeof(double) * (A->row_ptr[n] + 1));
  double* nB = (double*)malloc(sizeof(double) * (B->row_ptr[B->n] + 1));
  orc_block_norms(A, nA);
  orc_block_norms(B, nB);
  int64_t* offA = slot_offsets(A);
  int64_t* offB = slot_offsets(B);
  const int ncols = B->n;
  double* acc = (double*)calloc(ncols, sizeof(double));
  char* seen = (char*)calloc(ncols, 1);
  int* touched = (int*)malloc(sizeof(int) * (ncols + 1));
  int* pos = (int*)malloc(sizeof(int) * (ncols + 1));
  memset(C, 0, sizeof(*C));
  C->n = n;
  C->row_ptr = (int*)malloc(sizeof(int) * (n + 1));
  int cap = 1024, used = 0;
  C->col_ind = (int*)malloc(sizeof(int) * cap);
  C->row_ptr[0] = 0;
  /* symbolic */
  for (int i = 0; i < n; ++i) {
    int nt = 0;
    for (int a = A->row_ptr[i]; a < A->row_ptr[i + 1]; ++a) {
      const int kk = A->col_ind[a];
      for (int b = B->row_ptr[kk]; b < B->row_ptr[kk + 1]; ++b) {
        const int j = B->col_ind[b];
        if (upper && j < i) continue;
        if (!seen[j]) {
          seen[j] = 1;
          acc[j] = nA[a] * nB[b];
          touched[nt++] = j;
        } else {
          acc[j] += nA[a] * nB[b];
        }
      }
    }
    int kept = 0;
    for (int t = 0; t < nt; ++t) {
      const int j = touched[t];
      if (acc[j] > thr) touched[kept++] = j;
      seen[j] = 0;
    }
    qsort(touched, kept, sizeof(int), cmp_int);
    if (used + kept > cap) {
      while (used + kept > cap) cap *= 2;
      C->col_ind = (int*)realloc(C->col_ind, sizeof(int) * cap);
    }
    memcpy(C->col_ind + used, touched, sizeof(int) * kept);
    used += kept;
    C->row_ptr[i + 1] = used;
  }
  C->nnzb = used;
  C->stats[0] = used;
  /* value offsets of C */
  int64_t* offC = (int64_t*)malloc(sizeof(int64_t) * (used + 1));
  offC[0] = 0;
  for (int i = 0; i < n; ++i)
    for (int s = C->row_ptr[i]; s < C->row_ptr[i + 1]; ++s)
      offC[s + 1] = offC[s] + (int64_t)A->bsz[i] * B->bsz[C->col_ind[s]];
  C->nnz = offC[used];
  C->vals = (double*)calloc((size_t)C->nnz * cw + 1, sizeof(double));
  for (int j = 0; j < ncols; ++j) pos[j] = -1;
  int64_t products = 0, flops = 0;
  /* numeric */
  for (int i = 0; i < n; ++i) {
    for (int s = C->row_ptr[i]; s < C->row_ptr[i + 1]; ++s) pos[C->col_ind[s]] = s;
    const int r = A->bsz[i];
    const int row_count = A->row_ptr[i + 1] - A->row_ptr[i];
    const double row_eps = thr / (row_count > 1 ? row_count : 1);
    for (int a = A->row_ptr[i]; a < A->row_ptr[i + 1]; ++a) {
      const int kk = A->col_ind[a];
      const int inner = A->bsz[kk];
      const double* av = A->vals + offA[a] * cw;
      for (int b = B->row_ptr[kk]; b < B->row_ptr[kk + 1]; ++b) {
        if (nA[a] * nB[b] < row_eps) continue;
        const int j = B->col_ind[b];
        const int dst = pos[j];
        if (dst < 0) continue;
        const int c = B->bsz[j];
        const double* bv = B->vals + offB[b] * cw;
        double* cv = C->vals + offC[dst] * cw;
        ++products;
        flops += 2LL * r * inner * c * (cw == 2 ? 4 : 1);
        for (int t = 0; t < r; ++t)
          for (int q = 0; q < inner; ++q) {
            if (cw == 1) {
              const double x = av[t * inner + q];
              for (int u = 0; u < c; ++u) cv[t * c + u] = fma(x, bv[q * c + u], cv[t * c + u]);
            } else {
              const double xr = av[2 * (t * inner + q)], xi = av[2 * (t * inner + q) + 1];
              for (int u = 0; u < c; ++u) {
                const double br = bv[2 * (q * c + u)], bi = bv[2 * (q * c + u) + 1];
                cv[2 * (t * c + u)] += xr * br - xi * bi;
                cv[2 * (t * c + u) + 1] += xr * bi + xi * br;
              }
            }
          }
      }
    }
    for (int s = C->row_ptr[i]; s < C->row_ptr[i + 1]; ++s) pos[C->col_ind[s]] = -1;
  }
  C->stats[2] = products;
  C->stats[3] = flops;
  free(offC);
  filter_result(C, B->bsz, A->is_complex, thr);
  /* block sizes: rows from A, columns from B (square: same array) */
  C->stats[1] = C->nnzb;
  free(nA);
  free(nB);
  free(offA);
  free(offB);
  free(acc);
  free(seen);
  free(touched);
  free(pos);
}

void orc_spgemm(const orc_mat* A, const orc_mat* B, double thr, orc_result* C) { spgemm_impl(A, B, thr, 0, C); }

/* C = A B for a product known to be Hermitian (BlockSpMat::spmm_hermitian,
 * block_csr.hpp:1597-1617): U = the upper block triangle of the thresholded
 * product (spgemm_impl with upper), then C = U + strict_lower(U^H) -- row i
 * holds the conjugate transposes of U's blocks (k, i), k < i, in increasing
 * k, then U's blocks (i, j >= i) (conjugate_transpose with mirror,
 * ops/transpose.hpp:139-198) -- and every diagonal block is Hermitized:
 * d[r][c] = (d[r][c] + conj(d[c][r])) * 0.5 above the diagonal, its
 * conjugate below, the real part on it (hermitize_diagonal_blocks,
 * block_csr.hpp:1941-1966).  Stats: U's symbolic blocks, C's blocks, U's
 * products and flops. */
void orc_spgemm_hermitian(const orc_mat* A, const orc_mat* B, double thr, orc_result* C) {
  orc_result U;
  spgemm_impl(A, B, thr, 1, &U);
  const int n = U.n;
  const int cw = A->is_complex ? 2 : 1;
  const int* bsz = A->bsz;
  orc_mat uv = {n, bsz, U.row_ptr, U.col_ind, U.vals, A->is_complex};
  int64_t* offU = slot_offsets(&uv);
  /* column lists of U: for column i the slots (k, i), k ascending */
  int* cnt = (int*)calloc(n + 1, sizeof(int));
  for (int64_t s = 0; s < U.nnzb; ++s) cnt[U.col_ind[s] + 1]++;
  for (int j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
  int* cslot = (int*)malloc(sizeof(int) * (U.nnzb + 1));
  int* crow = (int*)malloc(sizeof(int) * (U.nnzb + 1));
  int* fill = (int*)malloc(sizeof(int) * (n + 1));
  memcpy(fill, cnt, sizeof(int) * (n + 1));
  for (int i = 0; i < n; ++i)
    for (int s = U.row_ptr[i]; s < U.row_ptr[i + 1]; ++s) {
      const int p = fill[U.col_ind[s]]++;
      cslot[p] = s;
      crow[p] = i;
    }
  memset(C, 0, sizeof(*C));
  C->n = n;
  C->row_ptr = (int*)malloc(sizeof(int) * (n + 1));
  C->col_ind = (int*)malloc(sizeof(int) * (2 * U.nnzb + 1));
  int* src = (int*)malloc(sizeof(int) * (2 * U.nnzb + 1));
  char* tr = (char*)malloc(2 * U.nnzb + 1);
  int64_t nb = 0;
  C->row_ptr[0] = 0;
  for (int i = 0; i < n; ++i) {
    for (int p = cnt[i]; p < cnt[i + 1]; ++p)
      if (crow[p] < i) {
        C->col_ind[nb] = crow[p];
        src[nb] = cslot[p];
        tr[nb++] = 1;
      }
    for (int s = U.row_ptr[i]; s < U.row_ptr[i + 1]; ++s)
      if (U.col_ind[s] >= i) {
        C->col_ind[nb] = U.col_ind[s];
        src[nb] = s;
        tr[nb++] = 0;
      }
    C->row_ptr[i + 1] = (int)nb;
  }
  C->nnzb = nb;
  orc_mat cv = {n, bsz, C->row_ptr, C->col_ind, NULL, A->is_complex};
  int64_t* offC = slot_offsets(&cv);
  C->nnz = offC[nb];
  C->vals = (double*)calloc((size_t)C->nnz * cw + 1, sizeof(double));
  for (int i = 0; i < n; ++i)
    for (int s = C->row_ptr[i]; s < C->row_ptr[i + 1]; ++s) {
      const int j = C->col_ind[s], ri = bsz[i], cj = bsz[j];
      const double* sv = U.vals + offU[src[s]] * cw;
      double* dv = C->vals + offC[s] * cw;
      for (int q = 0; q < ri; ++q)
        for (int t = 0; t < cj; ++t) {
          /* transposed: C(i, j)[q][t] = conj(U(j, i)[t][q]), U(j, i) is cj x ri */
          const int64_t e = tr[s] ? (int64_t)t * ri + q : (int64_t)q * cj + t;
          dv[(q * cj + t) * cw] = sv[e * cw];
          if (cw == 2) dv[(q * cj + t) * cw + 1] = tr[s] ? -sv[e * cw + 1] : sv[e * cw + 1];
        }
      if (j == i) {
        for (int r = 0; r < ri; ++r) {
          if (cw == 2) dv[(r * ri + r) * 2 + 1] = 0.0;
          for (int c = r + 1; c < ri; ++c) {
            double* up = dv + (r * ri + c) * cw;
            double* lo = dv + (c * ri + r) * cw;
            const double ar = (up[0] + lo[0]) * 0.5;
            up[0] = ar;
            lo[0] = ar;
            if (cw == 2) {
              const double ai = (up[1] - lo[1]) * 0.5;
              up[1] = ai;
              lo[1] = -ai;
            }
          }
        }
      }
    }
  C->stats[0] = U.stats[0];
  C->stats[1] = nb;
  C->stats[2] = U.stats[2];
  C->stats[3] = U.stats[3];
  free(offU);
  free(offC);
  free(cnt);
  free(cslot);
  free(crow);
  free(fill);
  free(src);
  free(tr);
  orc_result_free(&U);
}

/* Stand-alone filter on a copy (block_csr.hpp:1399). */
void orc_filter_blocks(const orc_mat* A, double thr, orc_result* C) {
  const int cw = A->is_complex ? 2 : 1;
  memset(C, 0, sizeof(*C));
  C->n = A->n;
  C->nnzb = A->row_ptr[A->n];
  int64_t* off = slot_offsets(A);
  C->nnz = off[C->nnzb];
  free(off);
  C->row_ptr = (int*)malloc(sizeof(int) * (A->n + 1));
  memcpy(C->row_ptr, A->row_ptr, sizeof(int) * (A->n + 1));
  C->col_ind = (int*)malloc(sizeof(int) * (C->nnzb + 1));
  memcpy(C->col_ind, A->col_ind, sizeof(int) * C->nnzb);
  C->vals = (double*)malloc(sizeof(double) * (C->nnz * cw + 1));
  memcpy(C->vals, A->vals, sizeof(double) * C->nnz * cw);
  filter_result(C, A->bsz, A->is_complex, thr);
}

/* Y <- alpha X + beta Y on the union pattern (ops/axpby.hpp:254 and its union
 * fallback); alpha/beta complex (re, im). */
void orc_axpby(const orc_mat* Y, double are, double aim, const orc_mat* X, double bre, double bim,
               orc_result* C) {
  const int cw = Y->is_complex ? 2 : 1;
  const int n = Y->n;
  int64_t* offY = slot_offsets(Y);
  int64_t* offX = slot_offsets(X);
  memset(C, 0, sizeof(*C));
  C->n = n;
  C->row_ptr = (int*)malloc(sizeof(int) * (n + 1));
  const int64_t cap = Y->row_ptr[n] + X->row_ptr[n] + 1;
  C->col_ind = (int*)malloc(sizeof(int) * cap);
  C->row_ptr[0] = 0;
  int64_t nb = 0;
  for (int i = 0; i < n; ++i) {
    int a = Y->row_ptr[i], b = X->row_ptr[i];
    while (a < Y->row_ptr[i + 1] || b < X->row_ptr[i + 1]) {
      const int ja = a < Y->row_ptr[i + 1] ? Y->col_ind[a] : 1 << 30;
      const int jb = b < X->row_ptr[i + 1] ? X->col_ind[b] : 1 << 30;
      const int j = ja < jb ? ja : jb;
      C->col_ind[nb++] = j;
      if (ja == j) ++a;
      if (jb == j) ++b;
    }
    C->row_ptr[i + 1] = (int)nb;
  }
  C->nnzb = nb;
  orc_mat cv = {n, Y->bsz, C->row_ptr, C->col_ind, NULL, Y->is_complex};
  int64_t* offC = slot_offsets(&cv);
  C->nnz = offC[nb];
  C->vals = (double*)calloc((size_t)C->nnz * cw + 1, sizeof(double));
  for (int i = 0; i < n; ++i) {
    int a = Y->row_ptr[i], b = X->row_ptr[i];
    for (int s = C->row_ptr[i]; s < C->row_ptr[i + 1]; ++s) {
      const int j = C->col_ind[s];
      const int64_t len = offC[s + 1] - offC[s];
      double* d = C->vals + offC[s] * cw;
      const int hy = a < Y->row_ptr[i + 1] && Y->col_ind[a] == j;
      const int hx = b < X->row_ptr[i + 1] && X->col_ind[b] == j;
      for (int64_t e = 0; e < len; ++e) {
        double yr = 0, yi = 0, xr = 0, xi = 0;
        if (hy) {
          yr = Y->vals[(offY[a] + e) * cw];
          if (cw == 2) yi = Y->vals[(offY[a] + e) * 2 + 1];
        }
        if (hx) {
          xr = X->vals[(offX[b] + e) * cw];
          if (cw == 2) xi = X->vals[(offX[b] + e) * 2 + 1];
        }
        if (cw == 1) {
          d[e] = are * xr + bre * yr;
        } else {
          d[2 * e] = are * xr - aim * xi + bre * yr - bim * yi;
          d[2 * e + 1] = are * xi + aim * xr + bre * yi + bim * yr;
        }
      }
      if (hy) ++a;
      if (hx) ++b;
    }
  }
  free(offY);
  free(offX);
  free(offC);
}

/* Conjugate transpose A^H (ops/transpose.hpp:179): block (j, i) of the
 * result is conj(A_ij)^T, rows of the result sorted by column. */
void orc_transpose(const orc_mat* A, orc_result* C) {
  const int cw = A->is_complex ? 2 : 1;
  const int n = A->n;
  const int64_t nnzb = A->row_ptr[n];
  int64_t* offA = slot_offsets(A);
  memset(C, 0, sizeof(*C));
  C->n = n;
  C->nnzb = nnzb;
  C->row_ptr = (int*)calloc(n + 1, sizeof(int));
  C->col_ind = (int*)malloc(sizeof(int) * (nnzb + 1));
  int* src = (int*)malloc(sizeof(int) * (nnzb + 1));
  for (int64_t s = 0; s < nnzb; ++s) C->row_ptr[A->col_ind[s] + 1]++;
  for (int j = 0; j < n; ++j) C->row_ptr[j + 1] += C->row_ptr[j];
  int* fill = (int*)malloc(sizeof(int) * (n + 1));
  memcpy(fill, C->row_ptr, sizeof(int) * (n + 1));
  for (int i = 0; i < n; ++i)
    for (int s = A->row_ptr[i]; s < A->row_ptr[i + 1]; ++s) {
      const int p = fill[A->col_ind[s]]++;
      C->col_ind[p] = i;
      src[p] = s;
    }
  orc_mat cv = {n, A->bsz, C->row_ptr, C->col_ind, NULL, A->is_complex};
  int64_t* offC = slot_offsets(&cv);
  C->nnz = offC[nnzb];
  C->vals = (double*)malloc(sizeof(double) * (C->nnz * cw + 1));
  for (int j = 0; j < n; ++j)
    for (int p = C->row_ptr[j]; p < C->row_ptr[j + 1]; ++p) {
      const int i = C->col_ind[p];
      const int s = src[p];
      const int r = A->bsz[i], c = A->bsz[j];
      const double* a = A->vals + offA[s] * cw;
      double* d = C->vals + offC[p] * cw;
      for (int t = 0; t < r; ++t)
        for (int q = 0; q < c; ++q) {
          /* d is c x r: d[q][t] = conj(a[t][q]) */
          if (cw == 1) {
            d[q * r + t] = a[t * c + q];
          } else {
            d[2 * (q * r + t)] = a[2 * (t * c + q)];
            d[2 * (q * r + t) + 1] = -a[2 * (t * c + q) + 1];
          }
        }
    }
  free(offA);
  free(offC);
  free(src);
  free(fill);
}

/* ------------------------------------------------ fused triple products */
/* Row accumulator of the fused executors (FusedRowAccumulator,
 * ops/spmm/common.hpp): columns in first-touch order, one r x c block and a
 * norm bound per column. */
typedef struct {
  int* pos;       /* column -> slot, -1 if untouched */
  int* cols;      /* touched columns, first-touch order */
  int64_t* voff;  /* value offset of each slot (in scalars) */
  double* bound;  /* per slot: sum of the pair norms that reached it */
  double* vals;
  int nt, cw;
  int64_t vused, vcap;
} orc_racc;

static void racc_init(orc_racc* a, int ncols, int cw) {
  a->pos = (int*)malloc(sizeof(int) * (ncols + 1));
  for (int j = 0; j < ncols; ++j) a->pos[j] = -1;
  a->cols = (int*)malloc(sizeof(int) * (ncols + 1));
  a->voff = (int64_t*)malloc(sizeof(int64_t) * (ncols + 1));
  a->bound = (double*)malloc(sizeof(double) * (ncols + 1));
  a->vcap = 1024;
  a->vals = (double*)malloc(sizeof(double) * a->vcap);
  a->nt = 0;
  a->vused = 0;
  a->cw = cw;
}

static void racc_free(orc_racc* a) {
  free(a->pos);
  free(a->cols);
  free(a->voff);
  free(a->bound);
  free(a->vals);
}

static void racc_clear(orc_racc* a) {
  for (int t = 0; t < a->nt; ++t) a->pos[a->cols[t]] = -1;
  a->nt = 0;
  a->vused = 0;
}

/* slot of column j (r x c block, zeroed when first touched) */
static int racc_obtain(orc_racc* a, int j, int r, int c) {
  if (a->pos[j] >= 0) return a->pos[j];
  const int64_t len = (int64_t)r * c * a->cw;
  if (a->vused + len > a->vcap) {
    while (a->vused + len > a->vcap) a->vcap *= 2;
    a->vals = (double*)realloc(a->vals, sizeof(double) * a->vcap);
  }
  const int s = a->nt++;
  a->cols[s] = j;
  a->voff[s] = a->vused;
  a->bound[s] = 0.0;
  memset(a->vals + a->vused, 0, sizeof(double) * len);
  a->vused += len;
  a->pos[j] = s;
  return s;
}

/* d (r x c) += x (r x m) y (m x c), row-major; complex interleaved */
static void block_mac(double* d, const double* x, const double* y, int r, int m, int c, int cw) {
  for (int t = 0; t < r; ++t)
    for (int q = 0; q < m; ++q) {
      if (cw == 1) {
        const double xv = x[t * m + q];
        for (int u = 0; u < c; ++u) d[t * c + u] = fma(xv, y[q * c + u], d[t * c + u]);
      } else {
        const double xr = x[2 * (t * m + q)], xi = x[2 * (t * m + q) + 1];
        for (int u = 0; u < c; ++u) {
          const double yr = y[2 * (q * c + u)], yi = y[2 * (q * c + u) + 1];
          d[2 * (t * c + u)] += xr * yr - xi * yi;
          d[2 * (t * c + u) + 1] += xr * yi + xi * yr;
        }
      }
    }
}

/* The finished row: blocks with Frobenius norm >= thr (all when thr <= 0),
 * columns ascending (stage_row_in_column_order, ops/spmm/common.hpp:1366). */
static void racc_stage(const orc_racc* a, int i, int r, const int* bsz, double thr, orc_result* C, int* order,
                       int64_t* vcap) {
  int kept = 0;
  for (int s = 0; s < a->nt; ++s) {
    const int64_t len = (int64_t)r * bsz[a->cols[s]] * a->cw;
    if (thr > 0.0) {
      double sq = 0.0;
      for (int64_t e = 0; e < len; ++e) sq += a->vals[a->voff[s] + e] * a->vals[a->voff[s] + e];
      if (sqrt(sq) < thr) continue;
    }
    order[kept++] = s;
  }
  /* insertion sort of the kept slots by column */
  for (int x = 1; x < kept; ++x) {
    const int v = order[x];
    int y = x - 1;
    while (y >= 0 && a->cols[order[y]] > a->cols[v]) {
      order[y + 1] = order[y];
      --y;
    }
    order[y + 1] = v;
  }
  for (int x = 0; x < kept; ++x) {
    const int s = order[x];
    const int64_t len = (int64_t)r * bsz[a->cols[s]] * a->cw;
    if (C->nnz * a->cw + len > *vcap) {
      while (C->nnz * a->cw + len > *vcap) *vcap *= 2;
      C->vals = (double*)realloc(C->vals, sizeof(double) * (*vcap));
    }
    C->col_ind = (int*)realloc(C->col_ind, sizeof(int) * (C->nnzb + 1));
    C->col_ind[C->nnzb++] = a->cols[s];
    memcpy(C->vals + C->nnz * a->cw, a->vals + a->voff[s], sizeof(double) * len);
    C->nnz += len / a->cw;
  }
  C->row_ptr[i + 1] = (int)C->nnzb;
}

static double max_block_norm(const double* norms, int64_t n) {
  double m = 0.0;
  for (int64_t s = 0; s < n; ++s)
    if (norms[s] > m) m = norms[s];
  return m;
}

/* A B A^H (rarh, A and B Hermitian) or A^H B A (rhar), upper block triangle,
 * one row at a time (RARhExecutor / RhARExecutor::fused_rows,
 * ops/spmm/rarh.hpp:190-330, ops/spmm/rhar.hpp:403-495):
 *  stage 1  T[i,:] = sum over the left factors of row i -- A's row i
 *           (rarh) or A's column i conjugate-transposed (rhar), in slot
 *           order, n_L of them -- times B's row k: a pair is skipped when
 *           |L_ik| |B_kl| < thr / (2 max(1, n_L) |B row k| max|A|)
 *           (0 when thr <= 0, max|A| = 0 or B's row is empty); T's columns
 *           in first-touch order, each with the sum of its pairs' norms;
 *  stage 2  C[i, j >= i] = sum over T's columns l (first-touch order) of
 *           T_il A_lj (A's row l), a pair skipped when
 *           bound(T_il) |A_lj| < thr / (2 |T row i|);
 *  drop     blocks with Frobenius norm < thr, columns ascending.
 * (rarh reads A^H's row l as A's row l: A Hermitian.) */
static void fused_rarh_impl(const orc_mat* A, const orc_mat* B, double thr, int rhar, orc_result* C) {
  const int n = A->n;
  const int cw = A->is_complex ? 2 : 1;
  const int64_t nnzbA = A->row_ptr[n];
  double* nA = (double*)malloc(sizeof(double) * (nnzbA + 1));
  double* nB = (double*)malloc(sizeof(double) * (B->row_ptr[B->n] + 1));
  orc_block_norms(A, nA);
  orc_block_norms(B, nB);
  const double amax = max_block_norm(nA, nnzbA);
  int64_t* offA = slot_offsets(A);
  int64_t* offB = slot_offsets(B);
  /* column view of A (rhar): per column i, the slots (k, i) by row k */
  int* cptr = (int*)calloc(n + 1, sizeof(int));
  int* cslot = (int*)malloc(sizeof(int) * (nnzbA + 1));
  int* crow = (int*)malloc(sizeof(int) * (nnzbA + 1));
  for (int64_t s = 0; s < nnzbA; ++s) cptr[A->col_ind[s] + 1]++;
  for (int j = 0; j < n; ++j) cptr[j + 1] += cptr[j];
  int* fill = (int*)malloc(sizeof(int) * (n + 1));
  memcpy(fill, cptr, sizeof(int) * (n + 1));
  for (int k = 0; k < n; ++k)
    for (int s = A->row_ptr[k]; s < A->row_ptr[k + 1]; ++s) {
      const int p = fill[A->col_ind[s]]++;
      cslot[p] = s;
      crow[p] = k;
    }
  double* lhs = (double*)malloc(sizeof(double) * 2 * 4096);
  orc_racc inner, outer;
  racc_init(&inner, n, cw);
  racc_init(&outer, n, cw);
  int* order = (int*)malloc(sizeof(int) * (n + 1));
  memset(C, 0, sizeof(*C));
  C->n = n;
  C->row_ptr = (int*)calloc(n + 1, sizeof(int));
  C->col_ind = (int*)malloc(sizeof(int));
  int64_t vcap = 1024;
  C->vals = (double*)malloc(sizeof(double) * vcap);
  int64_t products = 0;
  for (int i = 0; i < n; ++i) {
    const int r = A->bsz[i];
    racc_clear(&inner);
    racc_clear(&outer);
    const int nl = rhar ? cptr[i + 1] - cptr[i] : A->row_ptr[i + 1] - A->row_ptr[i];
    for (int e = 0; e < nl; ++e) {
      int k, s;
      if (rhar) {
        s = cslot[cptr[i] + e];
        k = crow[cptr[i] + e];
      } else {
        s = A->row_ptr[i] + e;
        k = A->col_ind[s];
      }
      const int m = A->bsz[k];
      const double* lb = A->vals + offA[s] * cw;
      if (rhar) {
        /* A[k,i] is m x r; the left factor is its conjugate transpose (r x m) */
        if ((int64_t)r * m > 4096) lhs = (double*)realloc(lhs, sizeof(double) * 2 * r * m);
        for (int t = 0; t < r; ++t)
          for (int q = 0; q < m; ++q) {
            if (cw == 1) {
              lhs[t * m + q] = lb[q * r + t];
            } else {
              lhs[2 * (t * m + q)] = lb[2 * (q * r + t)];
              lhs[2 * (t * m + q) + 1] = -lb[2 * (q * r + t) + 1];
            }
          }
        lb = lhs;
      }
      const int nbk = B->row_ptr[k + 1] - B->row_ptr[k];
      const double eps1 = (thr > 0.0 && amax > 0.0 && nbk > 0)
                              ? thr / (2.0 * (double)(nl > 1 ? nl : 1) * (double)nbk * amax)
                              : 0.0;
      for (int b = B->row_ptr[k]; b < B->row_ptr[k + 1]; ++b) {
        const double pair = nA[s] * nB[b];
        if (pair < eps1) continue;
        const int l = B->col_ind[b];
        const int c = B->bsz[l];
        const int slot = racc_obtain(&inner, l, r, c);
        inner.bound[slot] += pair;
        block_mac(inner.vals + inner.voff[slot], lb, B->vals + offB[b] * cw, r, m, c, cw);
        ++products;
      }
    }
    const double eps2 = (thr > 0.0 && inner.nt > 0) ? thr / (2.0 * (double)inner.nt) : 0.0;
    for (int t = 0; t < inner.nt; ++t) {
      const int l = inner.cols[t];
      const int m = A->bsz[l];
      for (int s = A->row_ptr[l]; s < A->row_ptr[l + 1]; ++s) {
        const int j = A->col_ind[s];
        if (j < i) continue;
        if (inner.bound[t] * nA[s] < eps2) continue;
        const int c = A->bsz[j];
        const int slot = racc_obtain(&outer, j, r, c);
        block_mac(outer.vals + outer.voff[slot], inner.vals + inner.voff[t], A->vals + offA[s] * cw, r, m, c, cw);
        ++products;
      }
    }
    racc_stage(&outer, i, r, A->bsz, thr, C, order, &vcap);
  }
  C->stats[0] = -1;
  C->stats[1] = C->nnzb;
  C->stats[2] = products;
  C->stats[3] = -1;
  racc_free(&inner);
  racc_free(&outer);
  free(order);
  free(lhs);
  free(fill);
  free(cptr);
  free(cslot);
  free(crow);
  free(offA);
  free(offB);
  free(nA);
  free(nB);
}

void orc_rarh_upper(const orc_mat* A, const orc_mat* B, double thr, orc_result* C) {
  fused_rarh_impl(A, B, thr, 0, C);
}

void orc_rhar_upper(const orc_mat* A, const orc_mat* B, double thr, orc_result* C) {
  fused_rarh_impl(A, B, thr, 1, C);
}

/* c2 A^2 + c1 A + c0 I, upper block triangle (A Hermitian), one row at a
 * time (SquarePolynomialExecutor::fused_rows,
 * ops/spmm/square_polynomial.hpp:115-265): pairs (i,k)(k,j), j >= i, skipped
 * when |A_ik| |A_kj| < thr / max(1, |A row i|) (0 when thr <= 0 or A has no
 * nonzero block); the accumulated row scaled by c2; then c1 A_ij added for
 * A's columns j >= i (reached even where no pair was) and c0 on the
 * diagonal block; blocks with norm < thr dropped, columns ascending.
 * Complex coefficients as (re, im). */
void orc_square_polynomial_upper(const orc_mat* A, double c2r, double c2i, double c1r, double c1i, double c0r,
                                 double c0i, double thr, orc_result* C) {
  const int n = A->n;
  const int cw = A->is_complex ? 2 : 1;
  const int64_t nnzbA = A->row_ptr[n];
  double* nA = (double*)malloc(sizeof(double) * (nnzbA + 1));
  orc_block_norms(A, nA);
  const int anz = max_block_norm(nA, nnzbA) > 0.0;
  int64_t* offA = slot_offsets(A);
  orc_racc acc;
  racc_init(&acc, n, cw);
  int* order = (int*)malloc(sizeof(int) * (n + 1));
  memset(C, 0, sizeof(*C));
  C->n = n;
  C->row_ptr = (int*)calloc(n + 1, sizeof(int));
  C->col_ind = (int*)malloc(sizeof(int));
  int64_t vcap = 1024;
  C->vals = (double*)malloc(sizeof(double) * vcap);
  int64_t products = 0;
  for (int i = 0; i < n; ++i) {
    const int r = A->bsz[i];
    racc_clear(&acc);
    const int cnt = A->row_ptr[i + 1] - A->row_ptr[i];
    const double eps = (thr > 0.0 && anz) ? thr / (double)(cnt > 1 ? cnt : 1) : 0.0;
    for (int a = A->row_ptr[i]; a < A->row_ptr[i + 1]; ++a) {
      const int k = A->col_ind[a];
      const int m = A->bsz[k];
      for (int b = A->row_ptr[k]; b < A->row_ptr[k + 1]; ++b) {
        const int j = A->col_ind[b];
        if (j < i) continue;
        if (nA[a] * nA[b] < eps) continue;
        const int c = A->bsz[j];
        const int slot = racc_obtain(&acc, j, r, c);
        block_mac(acc.vals + acc.voff[slot], A->vals + offA[a] * cw, A->vals + offA[b] * cw, r, m, c, cw);
        ++products;
      }
    }
    for (int s = 0; s < acc.nt; ++s) {
      const int64_t len = (int64_t)r * A->bsz[acc.cols[s]];
      double* d = acc.vals + acc.voff[s];
      for (int64_t e = 0; e < len; ++e) {
        if (cw == 1) {
          d[e] *= c2r;
        } else {
          const double xr = d[2 * e], xi = d[2 * e + 1];
          d[2 * e] = xr * c2r - xi * c2i;
          d[2 * e + 1] = xr * c2i + xi * c2r;
        }
      }
    }
    for (int a = A->row_ptr[i]; a < A->row_ptr[i + 1]; ++a) {
      const int j = A->col_ind[a];
      if (j < i) continue;
      const int c = A->bsz[j];
      const int slot = racc_obtain(&acc, j, r, c);
      double* d = acc.vals + acc.voff[slot];
      const double* src = A->vals + offA[a] * cw;
      for (int64_t e = 0; e < (int64_t)r * c; ++e) {
        if (cw == 1) {
          d[e] += c1r * src[e];
        } else {
          d[2 * e] += c1r * src[2 * e] - c1i * src[2 * e + 1];
          d[2 * e + 1] += c1r * src[2 * e + 1] + c1i * src[2 * e];
        }
      }
    }
    {
      const int slot = racc_obtain(&acc, i, r, r);
      double* d = acc.vals + acc.voff[slot];
      for (int t = 0; t < r; ++t) {
        d[(t * r + t) * cw] += c0r;
        if (cw == 2) d[(t * r + t) * 2 + 1] += c0i;
      }
    }
    racc_stage(&acc, i, r, A->bsz, thr, C, order, &vcap);
  }
  C->stats[0] = -1;
  C->stats[1] = C->nnzb;
  C->stats[2] = products;
  C->stats[3] = -1;
  racc_free(&acc);
  free(order);
  free(offA);
  free(nA);
}
