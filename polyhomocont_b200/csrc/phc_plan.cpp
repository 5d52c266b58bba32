// phc_plan.cpp -- compiles a packed sparse table (the components of
// type(sparse_system), src/sparse.f90:31-48) and the homotopy constants
// into the device table described in phc_internal.h.
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <map>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "phc_host.h"

namespace phc {

namespace {

struct Contribution {
  double cre, cim;
  int dest;
  int nf;             // factors in use
  int fac[kMaxN];     // power-table offsets e*N + j (at most N before reduction)
};

struct PackedRec {
  double cre, cim;
  uint64_t meta;
};

uint64_t pack_meta(int dest, int nf, unsigned flags, const int* fac) {
  uint64_t m = (uint64_t)(dest & 0x3ff) | ((uint64_t)(flags & 7) << 12);
  // unused factor slots stay 0, i.e. point at pw[0] = z_0^0 = 1, so that
  // every record multiplies three factors without branching
  for (int q = 0; q < nf; ++q) m |= (uint64_t)(fac[q] & 0x3ff) << (15 + 10 * q);
  return m;
}

// Contributions of all entries in one array, entry by entry (entry e owns
// cs[off[e] .. off[e+1]), in term order).
struct Entries {
  std::vector<int> off;
  std::vector<Contribution> cs;
  int count() const { return (int)off.size() - 1; }
  int size(int e) const { return off[e + 1] - off[e]; }
};

// Appends the records of one entry (its contributions in term order);
// every contribution has at most kMaxFac factors at this point.
void emit_entry(const Entries& E, int e, std::vector<PackedRec>& out) {
  for (int c = E.off[e]; c < E.off[e + 1]; ++c) {
    const Contribution& C = E.cs[c];
    const unsigned flags = (c + 1 == E.off[e + 1]) ? kRecLast : 0u;
    PackedRec r;
    r.cre = C.cre;
    r.cim = C.cim;
    r.meta = pack_meta(C.dest, C.nf, flags, C.fac);
    out.push_back(r);
  }
}

// Products with more than three factors: the first three are replaced by an
// extended power-table entry (shared between contributions with the same
// triple) until three or fewer remain. Entries are grouped in levels; an
// entry only uses table entries of lower levels.
struct PreTable {
  int base = 0;  // index of the first extended entry (pw_size)
  std::map<std::array<int, 3>, int> index;
  std::vector<std::array<int, 3>> entries;
  std::vector<int> level;
  int level_of(int f) const { return f >= base ? level[f - base] + 1 : 0; }
  int intern(const std::array<int, 3>& t) {
    auto it = index.find(t);
    if (it != index.end()) return it->second;
    const int e = base + (int)entries.size();
    entries.push_back(t);
    level.push_back(std::max(level_of(t[0]), std::max(level_of(t[1]), level_of(t[2]))));
    index[t] = e;
    return e;
  }
  // replaces the first three factors by their extended entry until at
  // most kMaxFac remain
  void reduce(int* fac, int& nf) {
    while (nf > kMaxFac) {
      const std::array<int, 3> t = {fac[0], fac[1], fac[2]};
      fac[0] = intern(t);
      std::memmove(fac + 1, fac + 3, sizeof(int) * (size_t)(nf - 3));
      nf -= 2;
    }
  }
};

// Longest-processing-time assignment of entries to the 32 lanes; each lane
// gets its entries in increasing entry order.
void schedule(const Entries& E, std::vector<std::vector<PackedRec>>& lanes) {
  const int ne = E.count();
  std::vector<long> cost(ne, 0);
  for (int e = 0; e < ne; ++e)
    for (int c = E.off[e]; c < E.off[e + 1]; ++c) cost[e] += 3 + (long)E.cs[c].nf;
  std::vector<int> order(ne);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return cost[a] > cost[b]; });
  long load[kWarp] = {}, recs[kWarp] = {};
  std::vector<int> lane_of(ne, -1);  // lane of each entry (-1: empty entry)
  for (int e : order) {
    if (E.size(e) == 0) continue;
    int best = 0;
    for (int l = 1; l < kWarp; ++l)
      if (load[l] < load[best]) best = l;
    load[best] += cost[e];
    lane_of[e] = best;
    recs[best] += E.size(e);
  }
  // The kernel runs every lane for the longest lane's record count rounded
  // up to a multiple of 4. If the LPT assignment misses the next lower
  // multiple of 4, try to pack the entries into lanes of that many records
  // (best fit, largest entries first); keep it when everything fits.
  long total = 0, lpt_max = 0;
  for (int l = 0; l < kWarp; ++l) {
    total += recs[l];
    lpt_max = std::max(lpt_max, recs[l]);
  }
  const long target = ((lpt_max + 3) & ~3L) - 4;
  if (target > 0 && target * kWarp >= total) {
    std::vector<int> by_size(order);
    std::stable_sort(by_size.begin(), by_size.end(),
                     [&](int a, int b) { return E.size(a) > E.size(b); });
    long fill[kWarp] = {};
    std::vector<int> packed(ne, -1);
    bool ok = true;
    for (int e : by_size) {
      const long sz = (long)E.size(e);
      if (sz == 0) continue;
      int best = -1;
      for (int l = 0; l < kWarp; ++l)
        if (fill[l] + sz <= target && (best < 0 || fill[l] > fill[best])) best = l;
      if (best < 0) {
        ok = false;
        break;
      }
      fill[best] += sz;
      packed[e] = best;
    }
    if (ok) {
      lane_of.swap(packed);
      for (int l = 0; l < kWarp; ++l) recs[l] = fill[l];
    }
  }
  lanes.assign(kWarp, {});
  for (int l = 0; l < kWarp; ++l) lanes[l].reserve((size_t)recs[l]);
  for (int e = 0; e < ne; ++e)
    if (lane_of[e] >= 0) emit_entry(E, e, lanes[lane_of[e]]);
}

// Writes one schedule's lane-interleaved arrays at the given offsets.
void store_schedule(const std::vector<std::vector<PackedRec>>& lanes, int len,
                    unsigned char* base, int off_d, int off_f, int off_m, int32_t* cnt) {
  double* cd = reinterpret_cast<double*>(base + off_d);
  float* cf = reinterpret_cast<float*>(base + off_f);
  uint64_t* cm = reinterpret_cast<uint64_t*>(base + off_m);
  for (int l = 0; l < kWarp; ++l) {
    cnt[l] = (int32_t)lanes[l].size();
    for (int i = 0; i < len; ++i) {
      const size_t slot = (size_t)i * kWarp + l;
      PackedRec r{0.0, 0.0, 0};
      if (i < (int)lanes[l].size()) r = lanes[l][i];
      cd[2 * slot] = r.cre;
      cd[2 * slot + 1] = r.cim;
      cf[2 * slot] = (float)r.cre;
      cf[2 * slot + 1] = (float)r.cim;
      cm[slot] = r.meta;
    }
  }
}

size_t max_len(const std::vector<std::vector<PackedRec>>& lanes) {
  size_t m = 0;
  for (const auto& v : lanes) m = std::max(m, v.size());
  return m;
}

}  // namespace

// Every index the kernels read out of a compiled table, checked on the host
// before the table is used: header sizes against the compile-time limits,
// array offsets against the table's size, each record's destination and
// power-table factors, the extended power-table levels (each entry built
// only from entries that exist before its level runs), and that no two
// records of a schedule finish the same entry. The kernels index shared
// memory with these values unchecked, so a table that fails here would make
// them read or write out of bounds; verify_plan turns that into an error
// status instead. It runs after every table compile (O(records)).
int verify_plan(const unsigned char* bytes, size_t size) {
  auto fail = [](const char* what) {
    set_last_error(std::string("table verification failed: ") + what);
    return PHC_ERR_UNSUPPORTED;
  };
  if (bytes == nullptr || size < sizeof(PlanHeader)) return fail("short table");
  PlanHeader H;
  std::memcpy(&H, bytes, sizeof(H));
  // (64-bit arithmetic throughout: a damaged header may hold any values)
  if (H.n < 1 || (int64_t)H.N != (int64_t)H.n + 1 || H.N > kMaxN) return fail("dimensions");
  if (H.S < H.N || H.S % 2 == 0 || (int64_t)H.n * H.S > 1024) return fail("row stride");
  if (H.maxexp < 1 || (int64_t)H.pw_size != ((int64_t)H.maxexp + 1) * H.N)
    return fail("power table size");
  if (H.n_pre < 0 || (int64_t)H.pw_total != (int64_t)H.pw_size + H.n_pre || H.pw_total > kMaxPw)
    return fail("extended power table size");
  if (H.n_levels < 0 || H.n_levels > kMaxLevels) return fail("levels");
  if (H.max_fac < 0 || H.max_fac > kMaxFac) return fail("factors per record");
  if (H.len_f < 0 || H.len_j < 0 || H.len_f % 4 || H.len_j % 4) return fail("schedule lengths");
  if (H.total_bytes < (int)sizeof(PlanHeader) || (size_t)H.total_bytes != size ||
      H.total_bytes % 16)
    return fail("table size");
  const int64_t sf = (int64_t)H.len_f * kWarp, sj = (int64_t)H.len_j * kWarp;
  auto region = [&](int32_t off, int64_t bytes_needed) {
    return off >= (int32_t)sizeof(PlanHeader) && off % 16 == 0 &&
           (int64_t)off + bytes_needed <= (int64_t)H.total_bytes;
  };
  if (!region(H.off_fd, sf * 16) || !region(H.off_ff, sf * 8) || !region(H.off_fm, sf * 8) ||
      !region(H.off_jd, sj * 16) || !region(H.off_jf, sj * 8) || !region(H.off_jm, sj * 8) ||
      !region(H.off_pre, (int64_t)H.n_pre * 8))
    return fail("array offsets");
  // kernels that evaluate only in FP64 stage the first bytes_fp64 bytes:
  // everything but the FP32 coefficients must lie there
  auto region64 = [&](int32_t off, int64_t bytes_needed) {
    return (int64_t)off + bytes_needed <= (int64_t)H.bytes_fp64;
  };
  if (H.bytes_fp64 < (int)sizeof(PlanHeader) || H.bytes_fp64 % 16 ||
      H.bytes_fp64 > H.total_bytes || !region64(H.off_fd, sf * 16) ||
      !region64(H.off_fm, sf * 8) || !region64(H.off_jd, sj * 16) ||
      !region64(H.off_jm, sj * 8) || !region64(H.off_pre, (int64_t)H.n_pre * 8))
    return fail("FP64 part of the table");
  int64_t radix = 1;
  for (int i = 0; i < H.n; ++i) {
    if (H.deg[i] < 1 || H.deg[i] - 1 > H.maxexp || H.radix[i] != radix) return fail("degrees");
    radix *= H.deg[i];
    if (radix > (int64_t)INT32_MAX) return fail("path count");
  }
  if (H.nstart != radix) return fail("path count");
  if (H.red_c < 0 || H.red_c >= H.N) return fail("patch pivot column");
  if (H.reduce != (reduce_patch_row(H.n) ? 1 : 0)) return fail("patch row elimination");
  // extended entries: level L may use plain entries and entries of levels < L
  std::vector<char> ready(H.pw_total, 0);
  std::fill(ready.begin(), ready.begin() + H.pw_size, 1);
  if (H.level_off[0] != 0 || H.level_off[H.n_levels] != 2 * H.n_pre)
    return fail("level ranges");
  const uint32_t* pre = reinterpret_cast<const uint32_t*>(bytes + H.off_pre);
  for (int L = 0; L < H.n_levels; ++L) {
    const int w0 = H.level_off[L], w1 = H.level_off[L + 1];
    if (w1 < w0 || (w1 - w0) % 2) return fail("level ranges");
    for (int w = w0; w < w1; w += 2) {
      const uint32_t t = pre[w], d = pre[w + 1];
      for (int q = 0; q < 3; ++q) {
        const uint32_t f = (t >> (10 * q)) & 0x3ffu;
        if (f >= (uint32_t)H.pw_total || !ready[f]) return fail("extended entry factor");
      }
      if (d < (uint32_t)H.pw_size || d >= (uint32_t)H.pw_total) return fail("extended entry");
    }
    for (int w = w0; w < w1; w += 2) ready[pre[w + 1]] = 1;
  }
  for (int e = H.pw_size; e < H.pw_total; ++e)
    if (!ready[e]) return fail("extended entry never computed");
  // records: destinations inside the Jacobian rows, factors inside the
  // computed table and within the kernel's schedule form, one finishing
  // record per entry
  auto check_schedule = [&](int len, int32_t off_m, const int32_t* cnt, bool jac) -> int {
    const uint64_t* meta = reinterpret_cast<const uint64_t*>(bytes + off_m);
    std::vector<char> finished((size_t)H.n * H.S, 0);
    for (int l = 0; l < kWarp; ++l) {
      if (cnt[l] < 0 || cnt[l] > len) return fail("records per lane");
      for (int i = 0; i < len; ++i) {
        const uint64_t m = meta[(size_t)i * kWarp + l];
        if (i >= cnt[l]) {
          if (m != 0) return fail("padding record");
          continue;
        }
        const int dest = (int)(m & 0x3ff);
        if (dest >= H.n * H.S || dest % H.S >= H.N) return fail("record destination");
        for (int q = 0; q < kMaxFac; ++q) {
          const int f = (int)((m >> (15 + 10 * q)) & 0x3ff);
          if (f >= H.pw_total) return fail("record factor");
          if (jac && q >= std::max(H.max_fac, 1) && f != 0) return fail("record schedule form");
        }
        if ((m >> 12) & kRecLast) {
          if (finished[dest]) return fail("entry finished twice");
          finished[dest] = 1;
        }
      }
    }
    return PHC_OK;
  };
  int st = check_schedule(H.len_f, H.off_fm, H.cnt_f, false);
  if (st == PHC_OK) st = check_schedule(H.len_j, H.off_jm, H.cnt_j, true);
  return st;
}

int validate_system(const phc_system* sys) {
  if (sys == nullptr) return PHC_ERR_INVALID_INPUT;
  const int n = sys->n;
  if (n < 1) return PHC_ERR_INVALID_INPUT;
  if (sys->first == nullptr || sys->deg == nullptr || sys->nterms < 0) return PHC_ERR_INVALID_INPUT;
  if (sys->nterms > 0 && (sys->hexps == nullptr || sys->coefs == nullptr))
    return PHC_ERR_INVALID_INPUT;
  if (sys->first[0] != 0 || sys->first[n] != sys->nterms) return PHC_ERR_INVALID_INPUT;
  for (int i = 0; i < n; ++i) {
    if (sys->first[i + 1] < sys->first[i]) return PHC_ERR_INVALID_INPUT;
    if (sys->deg[i] < 1) return PHC_ERR_INVALID_INPUT;
    for (int k = sys->first[i]; k < sys->first[i + 1]; ++k) {
      long sum = 0;
      for (int j = 0; j <= n; ++j) {
        const int e = sys->hexps[(size_t)k * (n + 1) + j];
        if (e < 0) return PHC_ERR_INVALID_INPUT;
        sum += e;
      }
      if (sum != sys->deg[i]) return PHC_ERR_INVALID_INPUT;  // homogeneous of degree d_i
    }
  }
  return PHC_OK;
}

// a / b by Smith's method (R. L. Smith, CACM 5 (1962) 435)
static std::complex<double> smith_div(std::complex<double> a, std::complex<double> b) {
  if (std::fabs(b.real()) < std::fabs(b.imag())) {
    const double ratio = b.real() / b.imag();
    const double den = b.real() * ratio + b.imag();
    return {(a.real() * ratio + a.imag()) / den, (a.imag() * ratio - a.real()) / den};
  }
  const double ratio = b.imag() / b.real();
  const double den = b.imag() * ratio + b.real();
  return {(a.imag() * ratio + a.real()) / den, (a.imag() - a.real() * ratio) / den};
}

int build_plan(const phc_system* sys, const phc_homotopy* hom, HostPlan* out) {
  int st = validate_system(sys);
  if (st != PHC_OK) return st;
  if (hom == nullptr || hom->b == nullptr || hom->patch == nullptr) return PHC_ERR_INVALID_INPUT;
  const int n = sys->n, N = n + 1;
  if (N > kMaxN) return PHC_ERR_UNSUPPORTED;
  // the power table also holds z_i^(d_i-1) and w^(d_i-1) of the start system
  int maxexp = 1;
  for (size_t q = 0; q < (size_t)sys->nterms * N; ++q) maxexp = std::max(maxexp, sys->hexps[q]);
  for (int i = 0; i < n; ++i) maxexp = std::max(maxexp, sys->deg[i] - 1);
  const int pw_size = (maxexp + 1) * N;
  if (pw_size > kMaxPw) return PHC_ERR_UNSUPPORTED;
  const int S = (N % 2 == 1) ? N : N + 1;

  PlanHeader H;
  std::memset(&H, 0, sizeof(H));
  H.n = n;
  H.N = N;
  H.S = S;
  H.maxexp = maxexp;
  H.pw_size = pw_size;
  int64_t radix = 1;
  for (int i = 0; i < n; ++i) {
    H.deg[i] = sys->deg[i];
    H.inv_deg[i] = 1.0 / (double)sys->deg[i];
    H.radix[i] = radix;
    radix *= sys->deg[i];
    if (radix > (int64_t)INT32_MAX) return PHC_ERR_INVALID_INPUT;
  }
  H.nstart = radix;
  H.gamma[0] = hom->gamma[0];
  H.gamma[1] = hom->gamma[1];
  for (int i = 0; i < n; ++i) {
    H.b[i][0] = hom->b[2 * i];
    H.b[i][1] = hom->b[2 * i + 1];
    H.argb[i] = std::atan2(H.b[i][1], H.b[i][0]);
  }
  for (int j = 0; j < N; ++j) {
    H.patch[j][0] = hom->patch[2 * j];
    H.patch[j][1] = hom->patch[2 * j + 1];
  }
  // the patch row is eliminated first on the device, pivoting on its
  // largest entry (first maximum of |a_j|)
  {
    int c = 0;
    double amax = -1.0, asum = 0.0;
    for (int j = 0; j < N; ++j) {
      const double m = std::hypot(H.patch[j][0], H.patch[j][1]);
      asum += m;
      if (m > amax) {
        amax = m;
        c = j;
      }
    }
    if (!(amax > 0.0)) return PHC_ERR_INVALID_INPUT;  // a zero patch
    H.reduce = reduce_patch_row(n) ? 1 : 0;
    H.red_c = c;
    H.patch_abs_sum = asum;
    const std::complex<double> ac(H.patch[c][0], H.patch[c][1]);
    const std::complex<double> inv = smith_div(std::complex<double>(1.0, 0.0), ac);
    H.inv_ac[0] = inv.real();
    H.inv_ac[1] = inv.imag();
    for (int j = 0; j < N; ++j) {
      const std::complex<double> r =
          smith_div(std::complex<double>(H.patch[j][0], H.patch[j][1]), ac);
      H.rho[j][0] = r.real();
      H.rho[j][1] = r.imag();
    }
  }

  // Jacobian contributions per entry, in term order (eval_terms,
  // src/sparse.f90:259-278). F^h itself is not tabulated: the kernel
  // obtains it from the Jacobian row by Euler's relation.
  // (two passes: count the contributions of each entry, then fill them in
  // term order into one array)
  Entries fent, jent;
  fent.off.assign(1, 0);
  const int ne = n * S;
  jent.off.assign((size_t)ne + 1, 0);
  for (int i = 0; i < n; ++i)
    for (int k = sys->first[i]; k < sys->first[i + 1]; ++k) {
      const int* e = sys->hexps + (size_t)k * N;
      for (int j = 0; j < N; ++j)
        if (e[j] > 0) ++jent.off[(size_t)i * S + j + 1];
    }
  for (int q = 0; q < ne; ++q) jent.off[q + 1] += jent.off[q];
  jent.cs.resize((size_t)jent.off[ne]);
  std::vector<int> fill(jent.off.begin(), jent.off.end() - 1);
  for (int i = 0; i < n; ++i) {
    for (int k = sys->first[i]; k < sys->first[i + 1]; ++k) {
      const int* e = sys->hexps + (size_t)k * N;
      const double cre = sys->coefs[2 * k], cim = sys->coefs[2 * k + 1];
      for (int j = 0; j < N; ++j) {
        if (e[j] <= 0) continue;
        Contribution& d = jent.cs[fill[(size_t)i * S + j]++];
        d.cre = (double)e[j] * cre;
        d.cim = (double)e[j] * cim;
        d.dest = i * S + j;
        d.nf = 0;
        if (e[j] > 1) d.fac[d.nf++] = (e[j] - 1) * N + j;
        for (int l = 0; l < N; ++l)
          if (l != j && e[l] > 0) d.fac[d.nf++] = e[l] * N + l;
      }
    }
  }
  PreTable pre;
  pre.base = pw_size;
  int max_fac = 0;
  for (auto& c : jent.cs) {
    pre.reduce(c.fac, c.nf);
    max_fac = std::max(max_fac, c.nf);
  }
  H.max_fac = max_fac;
  const int n_pre = (int)pre.entries.size();
  int n_levels = 0;
  for (int l : pre.level) n_levels = std::max(n_levels, l + 1);
  if (pw_size + n_pre > kMaxPw || n_levels > kMaxLevels) return PHC_ERR_UNSUPPORTED;
  // extended entries in level order (their indices are fixed already, so
  // the table lists (index, triple) per level)
  std::vector<uint32_t> pre_packed;
  H.n_pre = n_pre;
  H.n_levels = n_levels;
  H.pw_total = pw_size + n_pre;
  for (int L = 0; L < n_levels; ++L) {
    H.level_off[L] = (int32_t)pre_packed.size();
    for (int e = 0; e < n_pre; ++e) {
      if (pre.level[e] != L) continue;
      const auto& t = pre.entries[e];
      // 10 bits per factor + the 10-bit destination offset (e) in a second word
      pre_packed.push_back((uint32_t)(t[0] & 0x3ff) | ((uint32_t)(t[1] & 0x3ff) << 10) |
                           ((uint32_t)(t[2] & 0x3ff) << 20));
      pre_packed.push_back((uint32_t)(pw_size + e));
    }
  }
  H.level_off[n_levels] = (int32_t)pre_packed.size();
  std::vector<std::vector<PackedRec>> lf, lj;
  schedule(fent, lf);
  schedule(jent, lj);
  // lanes run the schedule in batches of four records
  const int len_f = (int)((max_len(lf) + 3) & ~(size_t)3);
  const int len_j = (int)((max_len(lj) + 3) & ~(size_t)3);
  H.len_f = len_f;
  H.len_j = len_j;
  size_t off = sizeof(PlanHeader);
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += (bytes + 15) & ~(size_t)15;
    return (int32_t)o;
  };
  const size_t sf = (size_t)len_f * kWarp, sj = (size_t)len_j * kWarp;
  H.off_fd = take(sf * 16);
  H.off_fm = take(sf * 8);
  H.off_jd = take(sj * 16);
  H.off_jm = take(sj * 8);
  H.off_pre = take(pre_packed.size() * 4);
  // the FP32 coefficients last: kernels that evaluate only in FP64 stage
  // the table without them
  H.bytes_fp64 = (int32_t)off;
  H.off_ff = take(sf * 8);
  H.off_jf = take(sj * 8);
  H.total_bytes = (int32_t)off;
  int nrec = 0;
  for (const auto& v : lf) nrec += (int)v.size();
  for (const auto& v : lj) nrec += (int)v.size();
  H.nrec = nrec;
  out->bytes.assign(off, 0);
  store_schedule(lf, len_f, out->bytes.data(), H.off_fd, H.off_ff, H.off_fm, H.cnt_f);
  store_schedule(lj, len_j, out->bytes.data(), H.off_jd, H.off_jf, H.off_jm, H.cnt_j);
  if (!pre_packed.empty())
    std::memcpy(out->bytes.data() + H.off_pre, pre_packed.data(), pre_packed.size() * 4);
  std::memcpy(out->bytes.data(), &H, sizeof(H));
  out->n = n;
  out->N = N;
  out->S = S;
  out->maxexp = maxexp;
  out->pw_size = pw_size + n_pre;
  out->nstart = radix;
  out->nrec = nrec;
  out->max_fac = max_fac;
  out->bytes_fp64 = H.bytes_fp64;
  return verify_plan(out->bytes.data(), out->bytes.size());
}

}  // namespace phc
