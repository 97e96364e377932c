// Symbolic tensor-operation patterns -> digital patterns, and the GEMM
// matricization permutations of the TAL-SH C ABI.
//
// talsh_get_contr_ptrn_str2dig keeps the behaviour of the reference
// (talshf.F90:619-667 with get_contr_pattern_dig, tensor_algebra_cpu.F90:5307-5531):
//  - tensors are "name(i1,i2,...)"; separators ',' or '|'; labels are
//    alphanumeric with an optional trailing '+' (contravariant, ignored for
//    matching); "name+(" conjugates that tensor (bit 0 D, bit 1 L, bit 2 R);
//  - a pattern without '*' is an addition/copy and gets an empty right tensor;
//    a trailing "*<scalar>" is dropped;
//  - digital value > 0: position in D; < 0: minus the position of the partner
//    index in the other input; an index in D, L and R is a hyper-index;
//  - the same non-zero error codes as the reference for malformed patterns.
// The implementation groups label occurrences in a table instead of editing a
// tagged string, but consumes them in the same left-to-right order, which is
// what makes the error codes order-dependent.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "common.h"

namespace tb {
namespace {

struct Occ {
  int arg;        // 0 D, 1 L, 2 R
  int pos;        // 1-based
  std::string label;
  bool used = false;
};

bool alnum(char c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9'); }

// Returns false for an invalid label; strips a trailing '+' into `label`.
bool parse_label(const char *b, int n, std::string &label) {
  if (n <= 0) return false;
  for (int j = 0; j < n; ++j) {
    if (alnum(b[j])) continue;
    if (b[j] == '+' && j == n - 1 && j > 0) { label.assign(b, n - 1); return true; }
    return false;
  }
  label.assign(b, n);
  return true;
}

int digitize(const std::string &s, int *dig, int &drank, int &lrank, int &rrank, int &conj) {
  size_t l = s.size();
  while (l > 0 && s[l - 1] == ' ') --l;
  if (l == 0) return 16;
  std::vector<Occ> occ;
  int ranks[3] = {0, 0, 0};
  int ntens = 0;
  conj = 0;
  size_t i = 0;
  while (i < l) {
    const size_t open = s.find('(', i);
    if (open == std::string::npos || open >= l) break;
    if (open >= 2 && s[open - 1] == '+' && (alnum(s[open - 2]) || s[open - 2] == '_')) conj |= 1 << ntens;
    if (ntens >= 3) return 1;
    const int t = ntens++;
    size_t lab_beg = open + 1;
    int pos = 0;
    bool closed = false, had_sep = false;
    for (i = open + 1; i < l; ++i) {
      const char c = s[i];
      if (c != ',' && c != '|' && c != ')') continue;
      const int len = (int)(i - lab_beg);
      if (c == ')' && len == 0) {
        if (had_sep) return 3;
        closed = true;
        ++i;
        break;
      }
      std::string lab;
      if (!parse_label(s.data() + lab_beg, len, lab)) return c == ')' ? 4 : 2;
      occ.push_back(Occ{t, ++pos, lab});
      if (c == ')') { closed = true; ++i; break; }
      had_sep = true;
      lab_beg = i + 1;
    }
    if (!closed) return 5;
    ranks[t] = pos;
  }
  if (ntens == 3) {
    drank = ranks[0]; lrank = ranks[1]; rrank = ranks[2];
    for (size_t a = 0; a < occ.size(); ++a) {
      if (occ[a].used) continue;
      const int k1 = occ[a].arg, k2 = occ[a].pos;
      size_t from = a + 1;
      for (int kf = 1; kf <= 2; ++kf) {
        size_t b = from;
        while (b < occ.size() && (occ[b].used || occ[b].label != occ[a].label)) ++b;
        if (b == occ.size()) {
          if (kf == 1) return 11;
          break;
        }
        const int k3 = occ[b].arg, k4 = occ[b].pos;
        if (k1 == 0 && k3 == 1) {
          if (kf != 1) return 8;
          dig[k4 - 1] = k2;
        } else if (k1 == 0 && k3 == 2) {
          dig[lrank + k4 - 1] = k2;
        } else if (k1 == 1 && k3 == 2) {
          if (kf != 1) return 9;
          dig[k2 - 1] = -k4;
          dig[lrank + k4 - 1] = -k2;
        } else {
          return 10;
        }
        occ[b].used = true;
      }
      occ[a].used = true;
    }
    return 0;
  }
  if (ntens == 2) {
    drank = ranks[0]; lrank = ranks[1];
    for (size_t a = 0; a < occ.size(); ++a) {
      if (occ[a].used) continue;
      size_t b = a + 1;
      while (b < occ.size() && (occ[b].used || occ[b].label != occ[a].label)) ++b;
      if (b == occ.size()) return 14;
      if (!(occ[a].arg == 0 && occ[b].arg == 1)) return 13;
      dig[occ[b].pos - 1] = occ[a].pos;
      occ[a].used = occ[b].used = true;
    }
    return 0;
  }
  return 15;
}

}  // namespace
}  // namespace tb

extern "C" int talsh_get_contr_ptrn_str2dig(const char *c_str, int *dig_ptrn, int *drank,
                                            int *lrank, int *rrank, int *conj_bits) {
  *drank = -1; *lrank = -1; *rrank = -1; *conj_bits = 0;
  if (c_str == nullptr) return -1;
  const size_t n = std::strlen(c_str);
  if (n > (size_t)MAX_CONTRACTION_PATTERN_LEN) return -1;
  std::string s(c_str, n);
  size_t star = s.find('*');
  if (star != std::string::npos && s.find('(', star) == std::string::npos) {
    s.resize(star);  // trailing scalar factor
    if (s.empty()) return -2;
    if (s.back() != ')') return -3;
    star = std::string::npos;
  }
  if (star == std::string::npos) s += "*R()";
  int dig[2 * MAX_TENSOR_RANK + 8];
  int dr = -1, lr = -1, rr = -1, cj = 0;
  const int rc = tb::digitize(s, dig, dr, lr, rr, cj);
  *drank = dr; *lrank = lr; *rrank = rr;  // ranks are reported even when matching fails
  if (rc) return rc;
  if (lr > MAX_TENSOR_RANK || rr > MAX_TENSOR_RANK || dr > MAX_TENSOR_RANK) return 1;
  for (int i = 0; i < lr + rr; ++i) dig_ptrn[i] = dig[i];
  *conj_bits = cj;
  return 0;
}

// Digital pattern -> symbolic pattern, the inverse direction (reference
// get_contr_pattern_sym, tensor_algebra_cpu.F90:5533-5611, called by talshc.cpp
// and talshxx.hpp): D's indices are named a, b, ... (one name per positive
// entry of the pattern, so a hyper-index is named twice), every contracted
// index of L takes the next free letter in order and its partner in R repeats
// that letter; '+' after a tensor name marks conjugation (bit 0 D, bit 1 L,
// bit 2 R).  The buffer must hold at most 15 + 4 * (rank_left + rank_right)
// characters plus the NUL; *cpl is the length without the NUL.  *ierr = 1 for
// a negative rank; also (the reference prints an undefined character or
// overruns there) for a rank above MAX_TENSOR_RANK or a contracted index of R
// whose partner position is not a contracted index of L.
extern "C" void get_contr_pattern_sym(const int *rank_left, const int *rank_right, const int *conj_bits,
                                      const int *cptrn_dig, char *cptrn_sym, int *cpl, int *ierr) {
  *ierr = 0;
  *cpl = 0;
  const int lr = *rank_left, rr = *rank_right, cj = *conj_bits;
  if (lr < 0 || rr < 0 || lr > MAX_TENSOR_RANK || rr > MAX_TENSOR_RANK) {
    *ierr = 1;
    return;
  }
  std::string s;
  const auto open = [&](char name, int bit) {
    s += name;
    if (cj & bit) s += '+';
    s += '(';
  };
  const auto close = [&] {
    if (s.back() == ',') s.back() = ')';
    else s += ')';
  };
  int nu = 0;
  for (int i = 0; i < lr + rr; ++i) nu += cptrn_dig[i] > 0;
  open('D', 1);
  for (int i = 0; i < nu; ++i) (s += char('a' + i)) += ',';
  close();
  s += "+=";
  open('L', 2);
  char label[MAX_TENSOR_RANK];
  int fresh = nu;
  for (int i = 0; i < lr; ++i) {
    const int v = cptrn_dig[i];
    label[i] = v > 0 ? char('a' + v - 1) : char('a' + fresh++);
    (s += label[i]) += ',';
  }
  close();
  s += '*';
  open('R', 4);
  for (int j = 0; j < rr; ++j) {
    const int v = cptrn_dig[lr + j];
    if (v > 0) {
      s += char('a' + v - 1);
    } else {
      if (-v < 1 || -v > lr || cptrn_dig[-v - 1] > 0) {
        *ierr = 1;
        return;
      }
      s += label[-v - 1];
    }
    s += ',';
  }
  close();
  std::memcpy(cptrn_sym, s.c_str(), s.size() + 1);
  *cpl = (int)s.size();
}

// ---------------------------------------------------------------------------
// Matricization permutations (GEMM 'T','N' by default).  These are exported
// for callers of the reference ABI; the GPU contraction of this core gathers
// operand tiles directly and does not use them.
// ---------------------------------------------------------------------------
namespace {

bool pattern_pairs_ok(int lrank, int rrank, const int *c, bool allow_hyper) {
  const int n = lrank + rrank;
  std::vector<int> uses(n + 2, 0);
  int unc = 0;
  for (int p = 1; p <= n; ++p) {
    const int v = c[p - 1];
    if (v < 0) {
      const bool left = p <= lrank;
      if (left ? (-v > rrank || c[lrank - v - 1] != -p) : (-v > lrank || c[-v - 1] != -(p - lrank)))
        return false;
    } else if (v > 0 && v <= n) {
      if (uses[v] == 0) { uses[v] = 1; ++unc; }
      else if (allow_hyper && p > lrank && uses[v] == 1) uses[v] = 2;
      else return false;
    } else {
      return false;
    }
  }
  for (int v = 1; v <= unc; ++v) if (uses[v] < 1) return false;
  return true;
}

// Stable sort of items 1..n (values in trn[1..n]) by key[item-1].
void stable_sort_items(int n, const int *key, int *trn) {
  std::vector<int> tmp(trn + 1, trn + 1 + n);
  std::stable_sort(tmp.begin(), tmp.end(), [&](int a, int b) { return key[a - 1] < key[b - 1]; });
  for (int i = 0; i < n; ++i) trn[i + 1] = tmp[i];
}

}  // namespace

extern "C" void get_contr_permutations(int gemm_tl, int gemm_tr, int lrank, int rrank,
                                       const int *cptrn, int conj_bits, int *dprm, int *lprm,
                                       int *rprm, int *ncd, int *nlu, int *nru, int *ierr) {
  *ierr = 0;
  if (lrank < 0 || rrank < 0 || !pattern_pairs_ok(lrank, rrank, cptrn, false)) { *ierr = 1; return; }
  bool lconj = conj_bits & 2, rconj = conj_bits & 4;
  if (conj_bits & 1) { lconj = !lconj; rconj = !rconj; }
  if (gemm_tl == 0 && lconj) { *ierr = 2; return; }
  // D: uncontracted indices of L then of R, kept in D order when both halves are already ordered.
  int dr = 0;
  dprm[0] = 1;
  for (int i = 0; i < lrank; ++i) if (cptrn[i] > 0) dprm[++dr] = cptrn[i];
  *nlu = dr;
  bool simple = dr >= 2;
  for (int i = 0; i < rrank; ++i) {
    const int v = cptrn[lrank + i];
    if (v > 0) { dprm[++dr] = v; if (v <= *nlu) simple = false; }
  }
  if (simple) for (int j = 1; j <= dr; ++j) dprm[j] = j;
  // R: contracted first (R order), then uncontracted.
  rprm[0] = 1; *nru = 0; *ncd = 0;
  if (rrank > 0) {
    int j = 0;
    for (int i = 0; i < rrank; ++i) if (cptrn[lrank + i] < 0) rprm[i + 1] = ++j;
    *ncd = j;
    *nru = rrank - j;
    for (int i = 0; i < rrank; ++i) {
      const int v = cptrn[lrank + i];
      if (v > 0) rprm[i + 1] = (simple && *nru >= 2) ? *ncd + (v - *nlu) : ++j;
    }
  }
  // L: contracted indices follow R's contracted order, then uncontracted.
  lprm[0] = 1;
  if (lrank > 0) {
    std::vector<int> key, who, ord(1, 1);
    for (int i = 0; i < lrank; ++i)
      if (cptrn[i] < 0) { who.push_back(i + 1); key.push_back(-cptrn[i]); ord.push_back((int)who.size()); }
    const int nc = (int)who.size();
    if (nc >= 2) stable_sort_items(nc, key.data(), ord.data());
    for (int p = 1; p <= nc; ++p) lprm[who[ord[p] - 1]] = p;
    int j = nc;
    for (int i = 0; i < lrank; ++i) {
      const int v = cptrn[i];
      if (v > 0) lprm[i + 1] = (simple && *nlu >= 2) ? *ncd + v : ++j;
    }
  }
  if (gemm_tl == 0)
    for (int i = 1; i <= lrank; ++i) lprm[i] = lprm[i] <= *ncd ? lprm[i] + *nlu : lprm[i] - *ncd;
  if (gemm_tr != 0 || rconj)
    for (int i = 1; i <= rrank; ++i) rprm[i] = rprm[i] <= *ncd ? rprm[i] + *nru : rprm[i] - *ncd;
}

extern "C" void get_contraction_permutations(int gemm_tl, int gemm_tr, int lrank, int rrank,
                                             const int *cptrn, int conj_bits, int *dprm,
                                             int *lprm, int *rprm, int *ncd, int *nlu, int *nru,
                                             int *nhu, int *ierr) {
  *ierr = 0; *ncd = 0; *nlu = 0; *nru = 0; *nhu = 0;
  dprm[0] = 1; lprm[0] = 1; rprm[0] = 1;
  if (!pattern_pairs_ok(lrank, rrank, cptrn, true)) { *ierr = 3; return; }
  if (lrank < 0 || rrank < 0) { *ierr = 1; return; }
  bool lconj = conj_bits & 2, rconj = conj_bits & 4;
  if (conj_bits & 1) { lconj = !lconj; rconj = !rconj; }
  if (gemm_tl == 0 && lconj) { *ierr = 2; return; }
  const int n = lrank + rrank;
  if (n > 0) {
    // Label every index: contracted -ncd..-1 (in L order), simple uncontracted
    // 1..ns in D order, hyper-indices after all D positions; sorting the labels
    // of each input yields its matricization.
    int dr = 0;
    std::vector<int> dcount(n + 2, 0);
    for (int i = 0; i < n; ++i) {
      const int v = cptrn[i];
      if (v > 0) { dr = std::max(dr, v); dcount[v]++; if (i < lrank) (*nlu)++; else (*nru)++; }
      else (*ncd)++;
    }
    *ncd /= 2;
    std::vector<int> dlab(dr + 2, 0);
    int simple = 0;
    for (int p = 1; p <= dr; ++p) {
      if (dcount[p] == 1) dlab[p] = ++simple;
      else if (dcount[p] == 2) dlab[p] = dr + ++(*nhu);
    }
    *nlu -= *nhu; *nru -= *nhu;
    std::vector<int> llab(lrank + 1), rlab(rrank + 1);
    int c = 0;
    for (int i = 1; i <= lrank; ++i) llab[i] = cptrn[i - 1] < 0 ? -(*ncd - c++) : dlab[cptrn[i - 1]];
    for (int i = 1; i <= rrank; ++i)
      rlab[i] = cptrn[lrank + i - 1] < 0 ? llab[-cptrn[lrank + i - 1]] : dlab[cptrn[lrank + i - 1]];
    std::vector<int> dnew;
    std::vector<int> ord;
    if (lrank > 0) {
      ord.assign(lrank + 1, 1);
      for (int i = 1; i <= lrank; ++i) ord[i] = i;
      stable_sort_items(lrank, llab.data() + 1, ord.data());
      for (int i = 1; i <= lrank; ++i) {
        const int o = ord[i];
        if (llab[o] >= 1 && llab[o] <= dr) dnew.push_back(llab[o]);
        lprm[o] = i;
      }
    }
    if (rrank > 0) {
      ord.assign(rrank + 1, 1);
      for (int i = 1; i <= rrank; ++i) ord[i] = i;
      stable_sort_items(rrank, rlab.data() + 1, ord.data());
      for (int i = 1; i <= rrank; ++i) {
        const int o = ord[i];
        if (rlab[o] >= 1 && rlab[o] <= dr) dnew.push_back(rlab[o]);
        else if (rlab[o] > dr) dnew.push_back((int)dnew.size() + 1);
        rprm[o] = i;
      }
    }
    for (int p = 1; p <= dr && p <= (int)dnew.size(); ++p) dprm[p] = dnew[p - 1];
  }
  if (gemm_tl == 0)
    for (int i = 1; i <= lrank; ++i) {
      if (lprm[i] <= *ncd) lprm[i] += *nlu;
      else if (lprm[i] <= *ncd + *nlu) lprm[i] -= *ncd;
    }
  if (gemm_tr != 0 || rconj)
    for (int i = 1; i <= rrank; ++i) {
      if (rprm[i] <= *ncd) rprm[i] += *nru;
      else if (rprm[i] <= *ncd + *nru) rprm[i] -= *ncd;
    }
}
