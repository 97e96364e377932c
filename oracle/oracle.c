/* Oracle for the talsh-b200 hot path -- TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Each routine restates the reference CPU algorithm it names.  The product
 * library never links this file; tests, smoke() and bench.py's CPU baseline do.
 */
#include "oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { float re, im; } c4_t;
typedef struct { double re, im; } c8_t;

static int kind_size(int kind) {
  switch (kind) {
    case 4: return 4;
    case 8: return 8;
    case 14: return 8;
    case 18: return 16;
    default: return 0;
  }
}
static int kind_is_complex(int kind) { return kind == 14 || kind == 18; }

/* ------------------------------------------------------------------------- */
/* Pattern parser: talshf.F90:619-667 (string preprocessing) and            */
/* tensor_algebra_cpu.F90:5307-5531 (get_contr_pattern_dig).                 */
/* ------------------------------------------------------------------------- */

typedef struct {
  int arg;      /* 0 = D, 1 = L, 2 = R */
  int pos;      /* 1-based position inside the tensor */
  int len;      /* label length (without a trailing '+') */
  const char *lab;
  int erased;
} orc_occ_t;

static int is_alnum_c(char c) {
  return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9');
}
static int is_alnum_underscore_c(char c) { return is_alnum_c(c) || c == '_'; }

/* index_label_ok (tensor_algebra_cpu.F90:5493-5521): alphanumeric, with an
 * optional trailing '+' (contravariant) that is not the first character. */
static int label_ok(const char *lb, int n, int *contra) {
  *contra = 0;
  if (n <= 0) return 0;
  for (int j = 0; j < n; ++j) {
    if (!is_alnum_c(lb[j])) {
      if (j < n - 1 || j == 0 || lb[j] != '+') return 0;
      *contra = 1;
    }
  }
  return 1;
}

static int same_label(const orc_occ_t *a, const orc_occ_t *b) {
  return a->len == b->len && memcmp(a->lab, b->lab, (size_t)a->len) == 0;
}

/* get_contr_pattern_dig restated over an occurrence list instead of a tagged string. */
static int contr_pattern_dig(const char *p, int l, int *drank, int *lrank, int *rrank, int *cptrn,
                             int *conj_bits) {
  orc_occ_t occ[3 * 100];
  int nocc = 0, adims[3] = {0, 0, 0};
  int n = -1, conj = 0, i = 0, ks = 0;
  *drank = -1; *lrank = -1; *rrank = -1;
  while (l > 0 && p[l - 1] == ' ') --l; /* len_trim */
  if (l <= 0) return 16;
  while (i < l) {
    while (p[i] != '(') { ++i; if (i >= l) goto done_scan; }
    if (i >= 2 && p[i - 1] == '+' && is_alnum_underscore_c(p[i - 2])) conj += (1 << (n + 1));
    ks = i; ++i; ++n;
    if (n > 2) return 1;
    int k = 1;
    int start = ks; /* index of the character before the current label */
    int seen_sep = 0;
    int closed = 0;
    while (i < l) {
      char c = p[i];
      if (c == ',' || c == '|') {
        int len = i - 1 - start, cv;
        if (!label_ok(p + start + 1, len, &cv)) return 2;
        if (nocc >= 300 || k > 99) return 2;
        occ[nocc].arg = n; occ[nocc].pos = k; occ[nocc].len = len - cv;
        occ[nocc].lab = p + start + 1; occ[nocc].erased = 0; ++nocc;
        start = i; seen_sep = 1; ++k;
      } else if (c == ')') {
        int len = i - 1 - start, cv;
        if (len <= 0) {
          if (seen_sep) return 3;
        } else {
          if (!label_ok(p + start + 1, len, &cv)) return 4;
          if (nocc >= 300 || k > 99) return 4;
          occ[nocc].arg = n; occ[nocc].pos = k; occ[nocc].len = len - cv;
          occ[nocc].lab = p + start + 1; occ[nocc].erased = 0; ++nocc;
          ++k;
        }
        ++i; closed = 1;
        break;
      }
      ++i;
    }
    if (!closed) return 5;
    adims[n] = k - 1;
  }
done_scan:
  if (n == 2) {
    *drank = adims[0]; *lrank = adims[1]; *rrank = adims[2];
    for (int t = 0; t < nocc; ++t) {
      if (occ[t].erased) continue;
      int k1 = occ[t].arg, k2 = occ[t].pos;
      for (int kf = 1; kf <= 2; ++kf) {
        int u = -1;
        for (int v = t + 1; v < nocc; ++v)
          if (!occ[v].erased && same_label(&occ[t], &occ[v])) { u = v; break; }
        if (u >= 0) {
          int k3 = occ[u].arg, k4 = occ[u].pos;
          if (k1 == 0 && k3 == 1) {
            if (kf != 1) return 8;
            cptrn[k4 - 1] = k2;
          } else if (k1 == 0 && k3 == 2) {
            cptrn[adims[1] + k4 - 1] = k2;
          } else if (k1 == 1 && k3 == 2) {
            if (kf != 1) return 9;
            cptrn[k2 - 1] = -k4;
            cptrn[adims[1] + k4 - 1] = -k2;
          } else {
            return 10;
          }
          occ[u].erased = 1;
        } else if (kf == 1) {
          return 11;
        }
      }
      occ[t].erased = 1;
    }
  } else if (n == 1) {
    *drank = adims[0]; *lrank = adims[1];
    for (int t = 0; t < nocc; ++t) {
      if (occ[t].erased) continue;
      int k1 = occ[t].arg, k2 = occ[t].pos;
      int u = -1;
      for (int v = t + 1; v < nocc; ++v)
        if (!occ[v].erased && same_label(&occ[t], &occ[v])) { u = v; break; }
      if (u < 0) return 14;
      if (k1 == 0 && occ[u].arg == 1) cptrn[occ[u].pos - 1] = k2; else return 13;
      occ[u].erased = 1; occ[t].erased = 1;
    }
  } else {
    return 15;
  }
  *conj_bits = conj;
  return 0;
}

int orc_str2dig(const char *s, int *dig, int *drank, int *lrank, int *rrank, int *conj_bits) {
  char buf[1024 + 8];
  int csl = 0, star = -1;
  int dgp[2 * ORC_MAX_RANK + 200];
  *drank = -1; *lrank = -1; *rrank = -1; *conj_bits = 0;
  while (s[csl] != '\0') {
    if (csl >= 1024) return -1;
    if (s[csl] == '*' && star < 0) star = csl;
    buf[csl] = s[csl];
    ++csl;
  }
  if (star >= 0) { /* "...*scalar": drop a trailing scalar factor */
    int has_paren = 0;
    for (int i = star; i < csl; ++i) if (buf[i] == '(') { has_paren = 1; break; }
    if (!has_paren) {
      csl = star; star = -1;
      if (csl <= 0) return -2;
      if (buf[csl - 1] != ')') return -3;
    }
  }
  if (star < 0) { memcpy(buf + csl, "*R()", 4); csl += 4; }
  if (csl > 0) {
    int ierr = contr_pattern_dig(buf, csl, drank, lrank, rrank, dgp, conj_bits);
    if (ierr != 0) return ierr;
    int dgl = *lrank + *rrank;
    for (int i = 0; i < dgl; ++i) dig[i] = dgp[i];
  }
  return 0;
}

/* get_contr_pattern_sym (tensor_algebra_cpu.F90:5533-5611): digital pattern ->
 * symbolic pattern, written position by position as the Fortran does (the
 * closing ')' replaces a trailing ',' or follows an empty '(').  Returns ierr:
 * 1 for a negative rank; also for a rank above ORC_MAX_RANK or an R index whose
 * partner is not a contracted L index (undefined in the reference). */
static void put_head(char *out, int *n, char name, int conj) {
  out[(*n)++] = name;
  if (conj) out[(*n)++] = '+';
  out[(*n)++] = '(';
}

static void put_close(char *out, int *n) {
  if (out[*n - 1] == '(') ++*n;
  out[*n - 1] = ')';
}

int orc_pattern_sym(int lrank, int rrank, int conj_bits, const int *dig, char *out, int *cpl) {
  char left_lbl[ORC_MAX_RANK];
  int n = 0, nu = 0, m;
  *cpl = 0;
  if (lrank < 0 || rrank < 0 || lrank > ORC_MAX_RANK || rrank > ORC_MAX_RANK) return 1;
  for (int i = 0; i < lrank + rrank; ++i) if (dig[i] > 0) ++nu;
  put_head(out, &n, 'D', conj_bits & 1);
  m = 'a';
  for (int i = 0; i < nu; ++i) { out[n++] = (char)m; out[n++] = ','; ++m; }
  put_close(out, &n);
  out[n++] = '+'; out[n++] = '=';
  put_head(out, &n, 'L', conj_bits & 2);
  for (int i = 0; i < lrank; ++i) {
    if (dig[i] > 0) {
      out[n++] = (char)('a' + dig[i] - 1);
    } else {
      left_lbl[i] = (char)m;
      out[n++] = (char)m;
      ++m;
    }
    out[n++] = ',';
  }
  put_close(out, &n);
  out[n++] = '*';
  put_head(out, &n, 'R', conj_bits & 4);
  for (int i = 0; i < rrank; ++i) {
    int v = dig[lrank + i];
    if (v > 0) {
      out[n++] = (char)('a' + v - 1);
    } else {
      if (-v < 1 || -v > lrank || dig[-v - 1] > 0) return 1;
      out[n++] = left_lbl[-v - 1];
    }
    out[n++] = ',';
  }
  put_close(out, &n);
  out[n] = '\0';
  *cpl = n;
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Permutation solvers                                                       */
/* ------------------------------------------------------------------------- */

/* merge_sort_key_int (combinatoric.F90:1316-1368): stable ascending sort of
 * trn[1..ni] (old item numbers) by key[old-1]. */
static void sort_by_key(int ni, const int *key, int *trn) {
  for (int a = 2; a <= ni; ++a) { /* insertion sort: stable, same order as a merge sort */
    int v = trn[a], b = a - 1;
    while (b >= 1 && key[trn[b] - 1] > key[v - 1]) { trn[b + 1] = trn[b]; --b; }
    trn[b + 1] = v;
  }
}

/* get_contraction_permutations (tensor_algebra_cpu.F90:5757-5956). */
int orc_contraction_permutations(int gemm_tl, int gemm_tr, int lrank, int rrank, const int *cptrn,
                                 int conj_bits, int *dprm, int *lprm, int *rprm, int *ncd,
                                 int *nlu, int *nru, int *nhu) {
  int n = lrank + rrank, drank = 0;
  int dtens[2 * ORC_MAX_RANK + 2] = {0}, ltens[ORC_MAX_RANK + 2] = {0}, rtens[ORC_MAX_RANK + 2] = {0};
  *ncd = 0; *nlu = 0; *nru = 0; *nhu = 0;
  dprm[0] = 1; lprm[0] = 1; rprm[0] = 1;
  /* contr_pattern_ok (:5916-5954) */
  if (n > 0) {
    int jd[2 * ORC_MAX_RANK + 2], jc = 0;
    for (int j = 1; j <= n; ++j) jd[j] = 0;
    for (int j0 = 1; j0 <= n; ++j0) {
      int j1 = cptrn[j0 - 1];
      if (j1 < 0) {
        if (j0 <= lrank) {
          if (-j1 > rrank) return 3;
          if (cptrn[lrank + (-j1) - 1] != -j0) return 3;
        } else {
          if (-j1 > lrank) return 3;
          if (cptrn[(-j1) - 1] != -(j0 - lrank)) return 3;
        }
      } else if (j1 > 0 && j1 <= n) {
        if (j0 <= lrank) {
          if (jd[j1] == 0) { jd[j1]++; jc++; } else return 3;
        } else {
          if (jd[j1] == 0) { jd[j1]++; jc++; } else if (jd[j1] == 1) jd[j1]++; else return 3;
        }
      } else {
        return 3;
      }
    }
    for (int j0 = 1; j0 <= jc; ++j0) if (jd[j0] != 1 && jd[j0] != 2) return 3;
  }
  if (lrank < 0 || rrank < 0) return 1;
  int left_conj = (conj_bits >> 1) & 1, right_conj = (conj_bits >> 2) & 1;
  if (conj_bits & 1) { left_conj = !left_conj; right_conj = !right_conj; }
  if (gemm_tl == 0 && left_conj) return 2;
  if (n > 0) {
    for (int i = 1; i <= n; ++i) dtens[i] = 0;
    for (int i = 1; i <= n; ++i) {
      int j = cptrn[i - 1];
      if (j > 0) {
        if (j > drank) drank = j;
        dtens[j]++;
        if (i <= lrank) (*nlu)++; else (*nru)++;
      } else if (j < 0) {
        (*ncd)++;
      }
    }
    *ncd /= 2;
    int j = 0;
    for (int i = 1; i <= drank; ++i) {
      if (dtens[i] == 1) { ++j; dtens[i] = j; }
      else if (dtens[i] == 2) { (*nhu)++; dtens[i] = drank + *nhu; }
    }
    *nlu -= *nhu; *nru -= *nhu;
    j = 0;
    for (int i = 1; i <= lrank; ++i) {
      if (cptrn[i - 1] < 0) { ltens[i] = -(*ncd - j); ++j; }
      else ltens[i] = dtens[cptrn[i - 1]];
    }
    for (int i = 1; i <= rrank; ++i) {
      if (cptrn[lrank + i - 1] < 0) rtens[i] = ltens[-cptrn[lrank + i - 1]];
      else rtens[i] = dtens[cptrn[lrank + i - 1]];
    }
    int k = 0, tmp[ORC_MAX_RANK + 2];
    if (lrank > 0) {
      for (int i = 0; i <= lrank; ++i) tmp[i] = (i == 0) ? 1 : i;
      if (lrank > 1) sort_by_key(lrank, ltens + 1, tmp);
      for (int i = 1; i <= lrank; ++i) {
        int o = tmp[i];
        if (ltens[o] >= 1 && ltens[o] <= drank) { ++k; dtens[k] = ltens[o]; }
      }
      for (int i = 1; i <= lrank; ++i) lprm[tmp[i]] = i; /* N2O -> O2N */
    }
    if (rrank > 0) {
      for (int i = 0; i <= rrank; ++i) tmp[i] = (i == 0) ? 1 : i;
      if (rrank > 1) sort_by_key(rrank, rtens + 1, tmp);
      for (int i = 1; i <= rrank; ++i) {
        int o = tmp[i];
        if (rtens[o] >= 1 && rtens[o] <= drank) { ++k; dtens[k] = rtens[o]; }
        else if (rtens[o] > drank) { ++k; dtens[k] = k; }
      }
      for (int i = 1; i <= rrank; ++i) rprm[tmp[i]] = i;
    }
    if (drank > 0) for (int i = 1; i <= drank; ++i) dprm[i] = dtens[i];
  }
  if (gemm_tl == 0) {
    for (int i = 1; i <= lrank; ++i) {
      if (lprm[i] <= *ncd) lprm[i] += *nlu;
      else if (lprm[i] <= *ncd + *nlu) lprm[i] -= *ncd;
    }
  }
  if (gemm_tr != 0 || right_conj) {
    for (int i = 1; i <= rrank; ++i) {
      if (rprm[i] <= *ncd) rprm[i] += *nru;
      else if (rprm[i] <= *ncd + *nru) rprm[i] -= *ncd;
    }
  }
  return 0;
}

/* get_contr_permutations (tensor_algebra_cpu.F90:5613-5755). */
int orc_contr_permutations(int gemm_tl, int gemm_tr, int lrank, int rrank, const int *cptrn,
                           int conj_bits, int *dprm, int *lprm, int *rprm, int *ncd, int *nlu,
                           int *nru) {
  int jl = lrank + rrank;
  int jkey[2 * ORC_MAX_RANK + 2], jtrn0[2 * ORC_MAX_RANK + 2], jtrn1[2 * ORC_MAX_RANK + 2];
  /* contr_pattern_ok (:5720-5753) */
  if (jl > 0) {
    int jc = 0;
    for (int j = 1; j <= jl; ++j) jkey[j] = 0;
    for (int j0 = 1; j0 <= jl; ++j0) {
      int j1 = cptrn[j0 - 1];
      if (j1 < 0) {
        if (j0 <= lrank) {
          if (-j1 > rrank || cptrn[lrank - j1 - 1] != -j0) return 1;
        } else {
          if (-j1 > lrank || cptrn[-j1 - 1] != -(j0 - lrank)) return 1;
        }
      } else if (j1 > 0 && j1 <= jl) {
        ++jc;
        if (jkey[j1] == 0) jkey[j1] = 1; else return 1;
      } else {
        return 1;
      }
    }
    for (int j0 = 1; j0 <= jc; ++j0) if (jkey[j0] != 1) return 1;
  }
  if (lrank < 0 || rrank < 0) return 1;
  int left_conj = (conj_bits >> 1) & 1, right_conj = (conj_bits >> 2) & 1;
  if (conj_bits & 1) { left_conj = !left_conj; right_conj = !right_conj; }
  if (gemm_tl == 0 && left_conj) return 2;
  int drank = 0, simple;
  dprm[0] = 1;
  for (int i = 1; i <= lrank; ++i) if (cptrn[i - 1] > 0) { ++drank; dprm[drank] = cptrn[i - 1]; }
  *nlu = drank;
  simple = (drank >= 2);
  for (int i = lrank + 1; i <= lrank + rrank; ++i) {
    if (cptrn[i - 1] > 0) {
      ++drank; dprm[drank] = cptrn[i - 1];
      if (cptrn[i - 1] <= *nlu) simple = 0;
    }
  }
  if (simple) for (int j = 1; j <= drank; ++j) dprm[j] = j;
  rprm[0] = 1; *nru = 0; *ncd = 0;
  if (rrank > 0) {
    int j = 0;
    for (int i = 1; i <= rrank; ++i) if (cptrn[lrank + i - 1] < 0) { ++j; rprm[i] = j; }
    *ncd = j;
    *nru = rrank - *ncd;
    if (simple && *nru >= 2) {
      for (int i = 1; i <= rrank; ++i)
        if (cptrn[lrank + i - 1] > 0) rprm[i] = *ncd + (cptrn[lrank + i - 1] - *nlu);
    } else {
      for (int i = 1; i <= rrank; ++i) if (cptrn[lrank + i - 1] > 0) { ++j; rprm[i] = j; }
    }
  }
  lprm[0] = 1;
  if (lrank > 0) {
    int j = 0;
    for (int i = 1; i <= lrank; ++i)
      if (cptrn[i - 1] < 0) { ++j; jtrn1[j] = i; jkey[j] = -cptrn[i - 1]; }
    for (int k = 0; k <= j; ++k) jtrn0[k] = (k == 0) ? 1 : k;
    if (j >= 2) sort_by_key(j, jkey + 1, jtrn0);
    for (int i = 1; i <= j; ++i) lprm[jtrn1[jtrn0[i]]] = i;
    if (simple && *nlu >= 2) {
      for (int i = 1; i <= lrank; ++i) if (cptrn[i - 1] > 0) lprm[i] = *ncd + cptrn[i - 1];
    } else {
      for (int i = 1; i <= lrank; ++i) if (cptrn[i - 1] > 0) { ++j; lprm[i] = j; }
    }
  }
  if (gemm_tl == 0) {
    for (int i = 1; i <= lrank; ++i) lprm[i] = (lprm[i] <= *ncd) ? lprm[i] + *nlu : lprm[i] - *ncd;
  }
  if (gemm_tr != 0 || right_conj) {
    for (int i = 1; i <= rrank; ++i) rprm[i] = (rprm[i] <= *ncd) ? rprm[i] + *nru : rprm[i] - *ncd;
  }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Permutation (transpose)                                                   */
/* ------------------------------------------------------------------------- */

static int perm_ok(int n, const int *o2n) {
  int seen[ORC_MAX_RANK + 1] = {0};
  for (int i = 0; i < n; ++i) {
    if (o2n[i] < 1 || o2n[i] > n || seen[o2n[i]]) return 0;
    seen[o2n[i]] = 1;
  }
  return 1;
}

static void copy_elem(int esize, const char *src, char *dst, int conj, int cplx) {
  memcpy(dst, src, (size_t)esize);
  if (conj && cplx) {
    if (esize == 8) { float *f = (float *)dst; f[1] = -f[1]; }
    else { double *d = (double *)dst; d[1] = -d[1]; }
  }
}

int orc_permute(int kind, int rank, const int *dims_in, const int *o2n, const void *in, void *out,
                int conj) {
  int esize = kind_size(kind);
  if (esize == 0 || rank < 0 || rank > ORC_MAX_RANK) return 1;
  if (rank > 0 && !perm_ok(rank, o2n)) return 2;
  size_t vol = 1, so[ORC_MAX_RANK];
  size_t dout[ORC_MAX_RANK];
  for (int i = 0; i < rank; ++i) { vol *= (size_t)dims_in[i]; dout[o2n[i] - 1] = (size_t)dims_in[i]; }
  size_t st[ORC_MAX_RANK];
  size_t s = 1;
  for (int k = 0; k < rank; ++k) { st[k] = s; s *= dout[k]; }
  for (int i = 0; i < rank; ++i) so[i] = st[o2n[i] - 1];
  size_t idx[ORC_MAX_RANK] = {0};
  size_t off_out = 0;
  const char *pin = (const char *)in;
  char *pout = (char *)out;
  int cplx = kind_is_complex(kind);
  for (size_t l = 0; l < vol; ++l) {
    copy_elem(esize, pin + l * esize, pout + off_out * esize, conj, cplx);
    for (int i = 0; i < rank; ++i) { /* odometer over input indices */
      if (++idx[i] < (size_t)dims_in[i]) { off_out += so[i]; break; }
      off_out -= so[i] * (idx[i] - 1);
      idx[i] = 0;
    }
  }
  return 0;
}

/* Cache-blocked transpose restating tensor_block_copy_dlf_r8 (tensor_algebra_cpu.F90:7699-7940):
 * minor input/output index sets bounded by a few cache lines, split dimensions, a
 * priority ordering of the combined minor set, and OpenMP over the external volume. */
#define BLK_BODY(T)                                                                               \
  do {                                                                                            \
    const T *tin = (const T *)in;                                                                 \
    T *tout = (T *)out;                                                                           \
    if (trivial) {                                                                                \
      _Pragma("omp parallel for schedule(guided) num_threads(nthreads)")                         \
      for (long long l0 = 0; l0 < (long long)bs; ++l0) tout[l0] = tin[l0];                        \
      break;                                                                                      \
    }                                                                                             \
    if (kf < n) {                                                                                 \
      long long segs[1025];                                                                       \
      long long bases_pri[ORC_MAX_RANK + 2];                                                      \
      int m = nthreads;                                                                           \
      segs[0] = 0;                                                                                \
      for (int t = 1; t <= m; ++t) segs[t] = segs[t - 1] + vol_ext / m + ((t - 1) < vol_ext % m); \
      long long l0b = 1;                                                                          \
      for (int i = kf + 1; i <= n; ++i) { bases_pri[ipr[i]] = l0b; l0b *= e[ipr[i]]; }            \
      _Pragma("omp parallel num_threads(nthreads)")                                              \
      {                                                                                           \
        int tid = 0;                                                                              \
        IF_OMP(tid = omp_get_thread_num();)                                                       \
        long long im[ORC_MAX_RANK + 2], db[ORC_MAX_RANK + 2], de[ORC_MAX_RANK + 2];               \
        for (int j = 1; j <= n; ++j) { db[j] = 0; de[j] = e[j] - 1; }                             \
        long long l2 = de[split_in], l3 = de[split_out], ls = bases_out[1];                       \
        for (long long l1 = 0; l1 <= l3; l1 += seg_out) {                                         \
          db[split_out] = l1; de[split_out] = (l1 + seg_out - 1 < l3) ? l1 + seg_out - 1 : l3;    \
          for (long long lq = 0; lq <= l2; lq += seg_in) {                                        \
            db[split_in] = lq; de[split_in] = (lq + seg_in - 1 < l2) ? lq + seg_in - 1 : l2;      \
            long long ll = segs[tid];                                                             \
            for (int i = n; i >= kf + 1; --i) { int j = ipr[i]; im[j] = ll / bases_pri[j]; ll -= im[j] * bases_pri[j]; } \
            long long vmin = 1;                                                                   \
            for (int i = 1; i <= kf; ++i) { int j = ipr[i]; vmin *= (de[j] - db[j] + 1); im[j] = db[j]; } \
            long long lin = 0, lout = 0;                                                          \
            for (int j = 1; j <= n; ++j) { lin += im[j] * bases_in[j]; lout += im[j] * bases_out[j]; } \
            long long le = de[1] - db[1], lb = (segs[tid + 1] - segs[tid]) * vmin;                \
            while (lb > 0) {                                                                      \
              for (long long q = 0; q <= le; ++q) tout[lout + q * ls] = tin[lin + q];             \
              lb -= le + 1;                                                                       \
              int adv = 0;                                                                        \
              for (int i = 2; i <= n; ++i) {                                                      \
                int j = ipr[i];                                                                   \
                if (im[j] < de[j]) { im[j]++; lin += bases_in[j]; lout += bases_out[j]; adv = 1; break; } \
                lin -= (im[j] - db[j]) * bases_in[j]; lout -= (im[j] - db[j]) * bases_out[j]; im[j] = db[j]; \
              }                                                                                   \
              if (!adv) break;                                                                    \
            }                                                                                     \
          }                                                                                       \
        }                                                                                         \
      }                                                                                           \
    } else {                                                                                      \
      long long l2 = e[split_in] - 1, l3 = e[split_out] - 1;                                      \
      long long nb0 = l2 / seg_in + 1, nb1 = l3 / seg_out + 1;                                    \
      _Pragma("omp parallel for schedule(dynamic) num_threads(nthreads)")                        \
      for (long long blk = 0; blk < nb0 * nb1; ++blk) {                                           \
        long long im[ORC_MAX_RANK + 2], db[ORC_MAX_RANK + 2], de[ORC_MAX_RANK + 2];               \
        for (int j = 1; j <= n; ++j) { db[j] = 0; de[j] = e[j] - 1; }                             \
        long long l1 = (blk / nb0) * seg_out, lq = (blk % nb0) * seg_in, ls = bases_out[1];       \
        db[split_out] = l1; de[split_out] = (l1 + seg_out - 1 < l3) ? l1 + seg_out - 1 : l3;      \
        db[split_in] = lq; de[split_in] = (lq + seg_in - 1 < l2) ? lq + seg_in - 1 : l2;          \
        long long vmin = 1;                                                                       \
        for (int i = 1; i <= kf; ++i) { int j = ipr[i]; vmin *= (de[j] - db[j] + 1); im[j] = db[j]; } \
        long long lin = 0, lout = 0;                                                              \
        for (int j = 1; j <= n; ++j) { lin += im[j] * bases_in[j]; lout += im[j] * bases_out[j]; } \
        long long le = de[1] - db[1], lb = vmin;                                                  \
        while (lb > 0) {                                                                          \
          for (long long q = 0; q <= le; ++q) tout[lout + q * ls] = tin[lin + q];                 \
          lb -= le + 1;                                                                           \
          int adv = 0;                                                                            \
          for (int i = 2; i <= n; ++i) {                                                          \
            int j = ipr[i];                                                                       \
            if (im[j] < de[j]) { im[j]++; lin += bases_in[j]; lout += bases_out[j]; adv = 1; break; } \
            lin -= (im[j] - db[j]) * bases_in[j]; lout -= (im[j] - db[j]) * bases_out[j]; im[j] = db[j]; \
          }                                                                                       \
          if (!adv) break;                                                                        \
        }                                                                                         \
      }                                                                                           \
    }                                                                                             \
  } while (0)

#ifdef _OPENMP
#define IF_OMP(x) x
#else
#define IF_OMP(x)
#endif

typedef struct { unsigned char b[16]; } b16_t;

int orc_permute_blocked(int kind, int rank, const int *dims_in, const int *o2n, const void *in,
                        void *out, int nthreads) {
  int esize = kind_size(kind);
  if (esize == 0 || rank < 1 || rank > ORC_MAX_RANK || !perm_ok(rank, o2n)) return 1;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 1024) nthreads = 1024;
  const int n = rank;
  long long e[ORC_MAX_RANK + 2], bases_in[ORC_MAX_RANK + 2], bases_out[ORC_MAX_RANK + 2];
  int trn[ORC_MAX_RANK + 2], n2o[ORC_MAX_RANK + 2], ipr[ORC_MAX_RANK + 2];
  for (int i = 1; i <= n; ++i) { e[i] = dims_in[i - 1]; trn[i] = o2n[i - 1]; }
  int trivial = 1;
  for (int i = 1; i <= n; ++i) if (trn[i] != i) { trivial = 0; break; }
  long long bs = 1;
  for (int i = 1; i <= n; ++i) { bases_in[i] = bs; bs *= e[i]; }
  bases_in[n + 1] = bs;
  for (int i = 1; i <= n; ++i) n2o[trn[i]] = i;
  n2o[n + 1] = n + 1;
  long long bo = 1;
  for (int i = 1; i <= n; ++i) { bases_out[n2o[i]] = bo; bo *= e[n2o[i]]; }
  bases_out[n + 1] = bo;
  const long long line = 64 / esize, cmin = 2 * line, clim = 4 * line;
  int kf = n, split_in = n, split_out = n;
  long long seg_in = e[n], seg_out = e[n];
  for (int j = 1; j <= n + 1; ++j) ipr[j] = j;
  if (!trivial && bs > 1024) {
    int k1, k2;
    for (k1 = 1; k1 <= n; ++k1) if (bases_in[k1 + 1] >= clim) break;
    k1 -= 1;
    for (k2 = 1; k2 <= n; ++k2) if (bases_out[n2o[k2 + 1]] >= clim) break;
    k2 -= 1;
    for (int j = k1 + 1; j <= n; ++j) { if (trn[j] <= k2) ++k1; else break; }
    for (int j = k2 + 1; j <= n; ++j) { if (n2o[j] <= k1) ++k2; else break; }
    int cin = bases_in[k1 + 1] < cmin, cout = bases_out[n2o[k2 + 1]] < cmin;
    if (cin && !cout) {
      ++k1; split_in = k1; seg_in = (clim - 1) / bases_in[split_in] + 1;
      split_out = n2o[k2]; seg_out = e[split_out];
    } else if (!cin && cout) {
      ++k2; split_in = n2o[k2]; seg_in = (clim - 1) / bases_out[split_in] + 1;
      split_out = k1; seg_out = e[split_out];
    } else if (cin && cout) {
      ++k1; ++k2;
      if (k1 == n2o[k2]) {
        long long mb = bases_in[k1] < bases_out[k1] ? bases_in[k1] : bases_out[k1];
        split_in = k1; seg_in = (clim - 1) / mb + 1; split_out = k1; seg_out = e[k1];
      } else {
        split_in = k1; seg_in = (clim - 1) / bases_in[k1] + 1;
        split_out = n2o[k2]; seg_out = (clim - 1) / bases_out[split_out] + 1;
      }
    } else {
      split_in = k1; seg_in = e[k1]; split_out = n2o[k2]; seg_out = e[split_out];
    }
    long long vol_min = 1;
    if (seg_in < e[split_in]) vol_min *= seg_in;
    if (seg_out < e[split_out]) vol_min *= seg_out;
    if (vol_min > 1) {
      for (int j = 1; j <= k1; ++j) if (j != split_in && j != split_out) vol_min *= e[j];
      for (int j = 1; j <= k2; ++j) {
        int l = n2o[j];
        if (l > k1 && l != split_in && l != split_out) vol_min *= e[l];
      }
      long long l = (clim * clim) / vol_min;
      if (l >= 2) {
        if (split_in == split_out) {
          seg_in *= l;
        } else if (l > 4) {
          l = (long long)sqrtf((float)l);
          seg_in = seg_in * l < e[split_in] ? seg_in * l : e[split_in];
          seg_out = seg_out * l < e[split_out] ? seg_out * l : e[split_out];
        } else {
          seg_in = seg_in * l < e[split_in] ? seg_in * l : e[split_in];
        }
      }
    }
    int l = 0;
    while (l < k1) { ++l; ipr[l] = l; if (bases_in[l + 1] >= cmin) break; }
    int m = l + 1, j = 0;
    while (j < k2) {
      ++j;
      int nn = n2o[j];
      if (nn >= m) { ++l; ipr[l] = nn; }
      if (bases_out[n2o[j + 1]] >= cmin) break;
    }
    int nq = j + 1;
    for (j = m; j <= k1; ++j) if (trn[j] >= nq) { ++l; ipr[l] = j; }
    for (j = nq; j <= k2; ++j) if (n2o[j] > k1) { ++l; ipr[l] = n2o[j]; }
    kf = l;
    for (j = k2 + 1; j <= n; ++j) if (n2o[j] > k1) { ++l; ipr[l] = n2o[j]; }
    ipr[n + 1] = n + 1;
    { /* the priority list must be a permutation with dimension 1 first */
      int seen[ORC_MAX_RANK + 2] = {0}, ok = (l == n && ipr[1] == 1);
      for (int q = 1; q <= n && ok; ++q) { if (ipr[q] < 1 || ipr[q] > n || seen[ipr[q]]) ok = 0; else seen[ipr[q]] = 1; }
      if (!ok) return orc_permute(kind, rank, dims_in, o2n, in, out, 0);
    }
  }
  long long vol_ext = 1;
  for (int j = kf + 1; j <= n; ++j) vol_ext *= e[ipr[j]];
  if (vol_ext < nthreads && kf < n) { /* too little external volume to share: use one thread */
    nthreads = (int)(vol_ext > 0 ? vol_ext : 1);
  }
  switch (esize) {
    case 4: BLK_BODY(float); break;
    case 8: BLK_BODY(double); break;
    case 16: BLK_BODY(b16_t); break;
  }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Copy / add / scale / init / norm                                          */
/* ------------------------------------------------------------------------- */

double orc_cmplx8_to_real8(double re, double im) {
  if (re != 0.0) return hypot(re, im) * (re > 0.0 ? 1.0 : -1.0);
  return im;
}

/* cpu_tensor_block_copy: transp = digital pattern (O2N); lconj = L-bit xor D-bit. */
int orc_tensor_copy(int kind, const int *cptrn, int rank, const int *ldims, const void *L, void *D,
                    int conj_bits) {
  int lconj = ((conj_bits >> 1) & 1) ^ (conj_bits & 1);
  if (rank == 0) {
    int es = kind_size(kind);
    copy_elem(es, (const char *)L, (char *)D, lconj, kind_is_complex(kind));
    return 0;
  }
  return orc_permute(kind, rank, ldims, cptrn, L, D, lconj);
}

/* Elementwise d = d + l*s in the data kind's own arithmetic, unfused, as
 * tensor_block_add does (tensor_algebra_cpu.F90:3412-3416, :3495-3500, :3578-3583). */
static void add_elems(int kind, size_t vol, void *D, const void *Lp, double sr, double si,
                      int lconj, int accum) {
  if (kind == 4) {
    float s = (float)orc_cmplx8_to_real8(sr, si);
    float *d = (float *)D; const float *l = (const float *)Lp;
    for (size_t i = 0; i < vol; ++i) { volatile float p = l[i] * s; d[i] = accum ? d[i] + p : p; }
  } else if (kind == 8) {
    double s = orc_cmplx8_to_real8(sr, si);
    double *d = (double *)D; const double *l = (const double *)Lp;
    for (size_t i = 0; i < vol; ++i) { volatile double p = l[i] * s; d[i] = accum ? d[i] + p : p; }
  } else if (kind == 14) {
    float ar = (float)sr, ai = (float)si;
    c4_t *d = (c4_t *)D; const c4_t *l = (const c4_t *)Lp;
    for (size_t i = 0; i < vol; ++i) {
      float xr = l[i].re, xi = lconj ? -l[i].im : l[i].im;
      volatile float t1 = xr * ar, t2 = xi * ai, t3 = xr * ai, t4 = xi * ar;
      volatile float pr = t1 - t2, pi = t3 + t4;
      if (accum) { d[i].re = d[i].re + pr; d[i].im = d[i].im + pi; }
      else { d[i].re = pr; d[i].im = pi; }
    }
  } else if (kind == 18) {
    c8_t *d = (c8_t *)D; const c8_t *l = (const c8_t *)Lp;
    for (size_t i = 0; i < vol; ++i) {
      double xr = l[i].re, xi = lconj ? -l[i].im : l[i].im;
      volatile double t1 = xr * sr, t2 = xi * si, t3 = xr * si, t4 = xi * sr;
      volatile double pr = t1 - t2, pi = t3 + t4;
      if (accum) { d[i].re = d[i].re + pr; d[i].im = d[i].im + pi; }
      else { d[i].re = pr; d[i].im = pi; }
    }
  }
}

/* cpu_tensor_block_add: permute L first when the pattern is not the identity,
 * then tensor_block_add (conj: D-bit flips the L-bit). */
int orc_tensor_add(int kind, const int *cptrn, int rank, const int *ldims, const void *L, void *D,
                   double sr, double si, int conj_bits) {
  int es = kind_size(kind);
  if (es == 0) return 1;
  int lconj = ((conj_bits >> 1) & 1) ^ (conj_bits & 1);
  if (!kind_is_complex(kind)) lconj = 0;
  size_t vol = 1;
  for (int i = 0; i < rank; ++i) vol *= (size_t)ldims[i];
  int permute = 0;
  for (int i = 0; i < rank; ++i) if (cptrn[i] != i + 1) { permute = 1; break; }
  const void *src = L;
  void *tmp = NULL;
  if (permute) {
    tmp = malloc(vol * (size_t)es);
    if (!tmp) return 2;
    int rc = orc_permute(kind, rank, ldims, cptrn, L, tmp, 0);
    if (rc) { free(tmp); return rc; }
    src = tmp;
  }
  add_elems(kind, vol, D, src, sr, si, lconj, 1);
  free(tmp);
  return 0;
}

/* The reference's multi-threaded add, as timed on the host cores: a
 * non-identity pattern first permutes L into a freshly allocated block with the
 * cache-blocked OpenMP transpose (cpu_tensor_block_add, talshf.F90:1857-1904,
 * calls tensor_block_copy and later destroys the block), then tensor_block_add
 * (tensor_algebra_cpu.F90:3312-3673) runs one OpenMP loop d = d + l*s, each
 * operation rounded on its own (the reference's GNU build has no FMA
 * contraction; this file is compiled with -ffp-contract=off).  Real kinds use
 * s = cmplx8_to_real8(alpha).  Result bit-identical to orc_tensor_add. */
int orc_tensor_add_blocked(int kind, int rank, const int *dims_in, const int *o2n, const void *L,
                           void *D, double sr, double si, int nthreads) {
  int es = kind_size(kind);
  if (es == 0 || rank < 1 || rank > ORC_MAX_RANK || !perm_ok(rank, o2n)) return 1;
  if (nthreads < 1) nthreads = 1;
  size_t vol = 1;
  for (int i = 0; i < rank; ++i) vol *= (size_t)dims_in[i];
  int permute = 0;
  for (int i = 0; i < rank; ++i) if (o2n[i] != i + 1) { permute = 1; break; }
  const void *src = L;
  void *tmp = NULL;
  if (permute) {
    tmp = malloc(vol * (size_t)es);
    if (!tmp) return 2;
    int rc = orc_permute_blocked(kind, rank, dims_in, o2n, L, tmp, nthreads);
    if (rc) { free(tmp); return rc; }
    src = tmp;
  }
  const long long n = (long long)vol;
  if (kind == 4) {
    const float s = (float)orc_cmplx8_to_real8(sr, si);
    float *d = (float *)D; const float *l = (const float *)src;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (long long i = 0; i < n; ++i) d[i] = d[i] + l[i] * s;
  } else if (kind == 8) {
    const double s = orc_cmplx8_to_real8(sr, si);
    double *d = (double *)D; const double *l = (const double *)src;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (long long i = 0; i < n; ++i) d[i] = d[i] + l[i] * s;
  } else if (kind == 14) {
    const float ar = (float)sr, ai = (float)si;
    c4_t *d = (c4_t *)D; const c4_t *l = (const c4_t *)src;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (long long i = 0; i < n; ++i) {
      const float pr = l[i].re * ar - l[i].im * ai, pi = l[i].re * ai + l[i].im * ar;
      d[i].re = d[i].re + pr; d[i].im = d[i].im + pi;
    }
  } else {
    c8_t *d = (c8_t *)D; const c8_t *l = (const c8_t *)src;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (long long i = 0; i < n; ++i) {
      const double pr = l[i].re * sr - l[i].im * si, pi = l[i].re * si + l[i].im * sr;
      d[i].re = d[i].re + pr; d[i].im = d[i].im + pi;
    }
  }
  free(tmp);
  return 0;
}

int orc_tensor_scale(int kind, size_t vol, void *D, double sr, double si, int conj_bits) {
  if (conj_bits & 1) si = -si;
  if (kind == 4) {
    float s = (float)orc_cmplx8_to_real8(sr, si); float *d = (float *)D;
    for (size_t i = 0; i < vol; ++i) d[i] = d[i] * s;
  } else if (kind == 8) {
    double s = orc_cmplx8_to_real8(sr, si); double *d = (double *)D;
    for (size_t i = 0; i < vol; ++i) d[i] = d[i] * s;
  } else if (kind == 14) {
    float ar = (float)sr, ai = (float)si; c4_t *d = (c4_t *)D;
    for (size_t i = 0; i < vol; ++i) {
      volatile float t1 = d[i].re * ar, t2 = d[i].im * ai, t3 = d[i].re * ai, t4 = d[i].im * ar;
      d[i].re = t1 - t2; d[i].im = t3 + t4;
    }
  } else if (kind == 18) {
    c8_t *d = (c8_t *)D;
    for (size_t i = 0; i < vol; ++i) {
      volatile double t1 = d[i].re * sr, t2 = d[i].im * si, t3 = d[i].re * si, t4 = d[i].im * sr;
      d[i].re = t1 - t2; d[i].im = t3 + t4;
    }
  } else {
    return 1;
  }
  return 0;
}

int orc_tensor_init(int kind, size_t vol, void *D, double sr, double si, int conj_bits) {
  if (conj_bits & 1) si = -si;
  if (kind == 4) { float *d = (float *)D; for (size_t i = 0; i < vol; ++i) d[i] = (float)sr; }
  else if (kind == 8) { double *d = (double *)D; for (size_t i = 0; i < vol; ++i) d[i] = sr; }
  else if (kind == 14) { c4_t *d = (c4_t *)D; for (size_t i = 0; i < vol; ++i) { d[i].re = (float)sr; d[i].im = (float)si; } }
  else if (kind == 18) { c8_t *d = (c8_t *)D; for (size_t i = 0; i < vol; ++i) { d[i].re = sr; d[i].im = si; } }
  else return 1;
  return 0;
}

double orc_norm1(int kind, size_t vol, const void *D) {
  double s = 0.0;
  if (kind == 4) { const float *d = (const float *)D; for (size_t i = 0; i < vol; ++i) s += (double)fabsf(d[i]); }
  else if (kind == 8) { const double *d = (const double *)D; for (size_t i = 0; i < vol; ++i) s += fabs(d[i]); }
  else if (kind == 14) { const c4_t *d = (const c4_t *)D; for (size_t i = 0; i < vol; ++i) s += (double)hypotf(d[i].re, d[i].im); }
  else if (kind == 18) { const c8_t *d = (const c8_t *)D; for (size_t i = 0; i < vol; ++i) s += hypot(d[i].re, d[i].im); }
  else return -1.0;
  return s;
}

/* ------------------------------------------------------------------------- */
/* Contraction                                                               */
/* ------------------------------------------------------------------------- */

static void load_c(int kind, const void *p, size_t i, double *re, double *im) {
  switch (kind) {
    case 4: *re = ((const float *)p)[i]; *im = 0.0; break;
    case 8: *re = ((const double *)p)[i]; *im = 0.0; break;
    case 14: *re = ((const c4_t *)p)[i].re; *im = ((const c4_t *)p)[i].im; break;
    default: *re = ((const c8_t *)p)[i].re; *im = ((const c8_t *)p)[i].im; break;
  }
}
static void store_c(int kind, void *p, size_t i, double re, double im) {
  switch (kind) {
    case 4: ((float *)p)[i] = (float)re; break;
    case 8: ((double *)p)[i] = re; break;
    case 14: ((c4_t *)p)[i].re = (float)re; ((c4_t *)p)[i].im = (float)im; break;
    default: ((c8_t *)p)[i].re = re; ((c8_t *)p)[i].im = im; break;
  }
}

static size_t vol_of(int rank, const int *dims) {
  size_t v = 1;
  for (int i = 0; i < rank; ++i) v *= (size_t)dims[i];
  return v;
}

int orc_tensor_contract(int kind, const int *cptrn, int drank, const int *ddims, int lrank,
                        const int *ldims, int rrank, const int *rdims, void *D, const void *L,
                        const void *R, double sr, double si, int conj_bits, int accumulative) {
  int es = kind_size(kind), cplx = kind_is_complex(kind);
  if (es == 0) return 1;
  /* contr_ptrn_ok (tensor_algebra_cpu.F90:4282-4348): extents and pairing */
  {
    int bus[3 * ORC_MAX_RANK + 3] = {0};
    int dr = drank, lr = lrank, rr = rrank;
    for (int j0 = 1; j0 <= lr; ++j0) {
      int j1 = cptrn[j0 - 1];
      if (j1 > 0 && j1 <= dr) {
        if (++bus[j1] > 1) return 8;
        bus[dr + j0]++;
        if (ldims[j0 - 1] != ddims[j1 - 1]) return 8;
      } else if (j1 < 0 && -j1 <= rr) {
        bus[dr + lr - j1]++;
        if (ldims[j0 - 1] != rdims[-j1 - 1]) return 8;
      } else return 8;
    }
    for (int j0 = lr + 1; j0 <= lr + rr; ++j0) {
      int j1 = cptrn[j0 - 1];
      if (j1 > 0 && j1 <= dr) {
        if (++bus[j1] > 2) return 8;
        bus[dr + j0]++;
        if (rdims[j0 - lr - 1] != ddims[j1 - 1]) return 8;
      } else if (j1 < 0 && -j1 <= lr) {
        bus[dr - j1]++;
        if (rdims[j0 - lr - 1] != ldims[-j1 - 1]) return 8;
      } else return 8;
    }
    for (int j0 = 1; j0 <= dr + lr + rr; ++j0)
      if (!(bus[j0] == 1 || (bus[j0] == 2 && j0 <= dr))) return 8;
  }
  int lconj = 0, rconj = 0;
  if (cplx) {
    lconj = (conj_bits >> 1) & 1; rconj = (conj_bits >> 2) & 1;
    if (conj_bits & 1) { lconj = !lconj; rconj = !rconj; }
  }
  double ar = sr, ai = si;
  size_t dvol = vol_of(drank, ddims), lvol = vol_of(lrank, ldims), rvol = vol_of(rrank, rdims);

  if (lrank == 0 && rrank == 0 && drank == 0) { /* MULTIPLY_SCALARS: d + (l*r)*alpha */
    double lre, lim, rre, rim, dre, dim;
    load_c(kind, L, 0, &lre, &lim); load_c(kind, R, 0, &rre, &rim); load_c(kind, D, 0, &dre, &dim);
    if (!accumulative) { dre = 0.0; dim = 0.0; }
    if (lconj) lim = -lim;
    if (rconj) rim = -rim;
    double pre = lre * rre - lim * rim, pim = lre * rim + lim * rre;
    double qre = pre * ar - pim * ai, qim = pre * ai + pim * ar;
    store_c(kind, D, 0, dre + qre, dim + qim);
    return 0;
  }
  if ((lrank == 0) != (rrank == 0)) {
    /* ADD_TENSOR: the tensor operand is permuted into D's order (its pattern
     * entries are D positions) and added with scale = scalar*alpha, using the
     * tensor_block_add rules (real kinds take cmplx8_to_real8 of the scale). */
    const void *T = lrank ? L : R;
    const void *S = lrank ? R : L;
    int tconj = lrank ? lconj : rconj, sconj = lrank ? rconj : lconj;
    int trank = lrank ? lrank : rrank;
    const int *tdims = lrank ? ldims : rdims;
    const int *tptrn = lrank ? cptrn : cptrn + lrank;
    double s_re, s_im;
    load_c(kind, S, 0, &s_re, &s_im);
    if (sconj) s_im = -s_im;
    double fr = s_re * ar - s_im * ai, fi = s_re * ai + s_im * ar; /* d_c8 * alf */
    int trivial = 1;
    for (int i = 0; i < trank; ++i) if (tptrn[i] != i + 1) { trivial = 0; break; }
    const void *src = T;
    void *tmp = NULL;
    if (!trivial) {
      tmp = malloc(dvol * (size_t)es);
      if (!tmp) return 2;
      orc_permute(kind, trank, tdims, tptrn, T, tmp, 0);
      src = tmp;
    }
    add_elems(kind, dvol, D, src, fr, fi, tconj, accumulative ? 1 : 0);
    free(tmp);
    return 0;
  }
  if (!accumulative) for (size_t i = 0; i < dvol; ++i) store_c(kind, D, i, 0.0, 0.0);
  if (!cplx) ai = 0.0; /* GEMM alpha of real kinds is real(alpha) */
  /* PARTIAL / FULL contraction through the CPU matricization */
  int dprm[ORC_MAX_RANK + 1], lprm[ORC_MAX_RANK + 1], rprm[ORC_MAX_RANK + 1], ncd, nlu, nru, nhu;
  int ierr = orc_contraction_permutations(1, 0, lrank, rrank, cptrn, cplx ? conj_bits : 0, dprm,
                                          lprm, rprm, &ncd, &nlu, &nru, &nhu);
  if (ierr) return 9;
  void *lt = malloc(lvol * es), *rt = malloc(rvol * es), *dt = malloc((dvol ? dvol : 1) * es);
  if (!lt || !rt || !dt) { free(lt); free(rt); free(dt); return 2; }
  orc_permute(kind, lrank, ldims, lprm + 1, L, lt, 0);
  orc_permute(kind, rrank, rdims, rprm + 1, R, rt, 0);
  int dn2o_o2n[ORC_MAX_RANK + 1];
  int dimsT[ORC_MAX_RANK + 1];
  if (drank > 0) {
    /* D is transposed to the matrix order with the inverse of dprm (N2O) */
    for (int k = 1; k <= drank; ++k) dn2o_o2n[dprm[k] - 1] = k;
    orc_permute(kind, drank, ddims, dn2o_o2n, D, dt, 0);
    for (int k = 1; k <= drank; ++k) dimsT[k - 1] = ddims[dprm[k] - 1];
  } else {
    memcpy(dt, D, (size_t)es);
  }
  /* matrix extents: D(lld, lrd, lhd) L(lcd, lld, lhd) R(lcd, lrd, lhd) or R(lrd, lcd, lhd) */
  size_t lcd = 1, lld = 1, lrd = 1, lhd = 1;
  {
    int pos = 0;
    int lperm_dims[ORC_MAX_RANK];
    for (int i = 0; i < lrank; ++i) lperm_dims[lprm[i + 1] - 1] = ldims[i];
    for (int i = 0; i < ncd; ++i) lcd *= (size_t)lperm_dims[pos++];
    for (int i = 0; i < nlu; ++i) lld *= (size_t)lperm_dims[pos++];
    for (int i = 0; i < nhu; ++i) lhd *= (size_t)lperm_dims[pos++];
    int rperm_dims[ORC_MAX_RANK];
    for (int i = 0; i < rrank; ++i) rperm_dims[rprm[i + 1] - 1] = rdims[i];
    size_t rv = 1;
    for (int i = 0; i < ncd + nru; ++i) rv *= (size_t)rperm_dims[i];
    lrd = rv / (lcd ? lcd : 1);
  }
  for (size_t h = 0; h < lhd; ++h) {
    for (size_t j = 0; j < lrd; ++j) {
      for (size_t i = 0; i < lld; ++i) {
        double acc_re = 0.0, acc_im = 0.0;
        for (size_t c = 0; c < lcd; ++c) {
          double a_re, a_im, b_re, b_im;
          load_c(kind, lt, c + lcd * (i + lld * h), &a_re, &a_im);
          if (!rconj) load_c(kind, rt, c + lcd * (j + lrd * h), &b_re, &b_im);
          else load_c(kind, rt, j + lrd * (c + lcd * h), &b_re, &b_im);
          if (lconj) a_im = -a_im;
          if (rconj) b_im = -b_im;
          acc_re += a_re * b_re - a_im * b_im;
          acc_im += a_re * b_im + a_im * b_re;
        }
        double vr = acc_re * ar - acc_im * ai, vi = acc_re * ai + acc_im * ar;
        size_t di = i + lld * (j + lrd * h);
        double d_re, d_im;
        load_c(kind, dt, di, &d_re, &d_im);
        store_c(kind, dt, di, d_re + vr, d_im + vi);
      }
    }
  }
  if (drank > 0) {
    int o2n[ORC_MAX_RANK];
    for (int k = 1; k <= drank; ++k) o2n[k - 1] = dprm[k]; /* back-transpose with do2n */
    orc_permute(kind, drank, dimsT, o2n, dt, D, 0);
  } else {
    memcpy(D, dt, (size_t)es);
  }
  free(lt); free(rt); free(dt);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Slicing / insertion (tensor_algebra_cpu.F90:6900-6974, :7216-7290)          */
/* ------------------------------------------------------------------------- */
/* One element: d = d*beta + s*alpha in the element's own precision, complex
 * products written out as the Fortran complex multiply does them. */
#define ORC_SLICE_MOVE_REAL(T)                                                   \
  {                                                                              \
    T *dp = (T *)dst + di;                                                       \
    const T sv = ((const T *)src)[si];                                           \
    *dp = *dp * (T)bet + sv * (T)1;                                              \
  }
#define ORC_SLICE_MOVE_CPLX(CT, T)                                               \
  {                                                                              \
    CT *dp = (CT *)dst + di;                                                     \
    const CT sv = ((const CT *)src)[si];                                         \
    const T bre = (T)bet, one = (T)1, zero = (T)0;                               \
    const T pre = dp->re * bre - dp->im * zero, pim = dp->re * zero + dp->im * bre; \
    const T qre = sv.re * one - sv.im * zero, qim = sv.re * zero + sv.im * one; \
    dp->re = pre + qre;                                                          \
    dp->im = pim + qim;                                                          \
  }

static int orc_slice_move(int insert, int kind, int rank, const int *full_dims, const int *slice_dims,
                          const int *offsets, const void *src, void *dst, int accumulative) {
  if (kind_size(kind) == 0 || rank < 1 || rank > ORC_MAX_RANK) return 1;
  for (int i = 0; i < rank; ++i)
    if (full_dims[i] <= 0 || slice_dims[i] <= 0 || offsets[i] < 0 || offsets[i] + slice_dims[i] > full_dims[i])
      return 1;
  const double bet = accumulative ? 1.0 : 0.0;
  size_t fstr[ORC_MAX_RANK], svol = 1, s = 1;
  for (int i = 0; i < rank; ++i) { fstr[i] = s; s *= (size_t)full_dims[i]; svol *= (size_t)slice_dims[i]; }
  int im[ORC_MAX_RANK] = {0};
  for (size_t e = 0; e < svol; ++e) {
    size_t f = 0;
    for (int i = 0; i < rank; ++i) f += (size_t)(offsets[i] + im[i]) * fstr[i];
    const size_t si = insert ? e : f, di = insert ? f : e;
    switch (kind) {
      case 4: ORC_SLICE_MOVE_REAL(float) break;
      case 8: ORC_SLICE_MOVE_REAL(double) break;
      case 14: ORC_SLICE_MOVE_CPLX(c4_t, float) break;
      default: ORC_SLICE_MOVE_CPLX(c8_t, double) break;
    }
    for (int i = 0; i < rank; ++i) {
      if (++im[i] < slice_dims[i]) break;
      im[i] = 0;
    }
  }
  return 0;
}

int orc_tensor_slice(int kind, int rank, const int *full_dims, const int *slice_dims, const int *offsets,
                     const void *full, void *slice, int accumulative) {
  return orc_slice_move(0, kind, rank, full_dims, slice_dims, offsets, full, slice, accumulative);
}

int orc_tensor_insert(int kind, int rank, const int *full_dims, const int *slice_dims, const int *offsets,
                      const void *slice, void *full, int accumulative) {
  return orc_slice_move(1, kind, rank, full_dims, slice_dims, offsets, slice, full, accumulative);
}

/* ------------------------------------------------------------------------- */
/* Generator: mt19937_64                                                     */
/* ------------------------------------------------------------------------- */
typedef struct { uint64_t mt[312]; int mti; } orc_mt64_t;

static void mt64_seed(orc_mt64_t *g, uint64_t seed) {
  g->mt[0] = seed;
  for (int i = 1; i < 312; ++i)
    g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
  g->mti = 312;
}
static uint64_t mt64_next(orc_mt64_t *g) {
  static const uint64_t mag01[2] = {0ULL, 0xB5026F5AA96619E9ULL};
  const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL;
  if (g->mti >= 312) {
    int i;
    uint64_t x;
    for (i = 0; i < 312 - 156; ++i) {
      x = (g->mt[i] & UM) | (g->mt[i + 1] & LM);
      g->mt[i] = g->mt[i + 156] ^ (x >> 1) ^ mag01[(int)(x & 1ULL)];
    }
    for (; i < 311; ++i) {
      x = (g->mt[i] & UM) | (g->mt[i + 1] & LM);
      g->mt[i] = g->mt[i + (156 - 312)] ^ (x >> 1) ^ mag01[(int)(x & 1ULL)];
    }
    x = (g->mt[311] & UM) | (g->mt[0] & LM);
    g->mt[311] = g->mt[155] ^ (x >> 1) ^ mag01[(int)(x & 1ULL)];
    g->mti = 0;
  }
  uint64_t x = g->mt[g->mti++];
  x ^= (x >> 29) & 0x5555555555555555ULL;
  x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
  x ^= (x << 37) & 0xFFF7EEE000000000ULL;
  x ^= (x >> 43);
  return x;
}

void orc_fill_uniform(int kind, size_t vol, void *out, unsigned long long seed) {
  orc_mt64_t g;
  mt64_seed(&g, (uint64_t)seed);
  size_t n = vol * (kind_is_complex(kind) ? 2 : 1);
  for (size_t i = 0; i < n; ++i) {
    double u = 2.0 * (double)(mt64_next(&g) >> 11) * (1.0 / 9007199254740992.0) - 1.0;
    if (kind == 4 || kind == 14) ((float *)out)[i] = (float)u;
    else ((double *)out)[i] = u;
  }
}
