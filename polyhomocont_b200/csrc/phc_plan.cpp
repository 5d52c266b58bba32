// phc_plan.cpp -- compiles a packed sparse table (the components of
// type(sparse_system), src/sparse.f90:31-48) and the homotopy constants
// into the device table described in phc_internal.h.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "phc_host.h"

namespace phc {

namespace {

struct Contribution {
  double cre, cim;
  int dest;
  std::vector<int> fac;  // power-table offsets e*N + j
};

// Appends the records of one entry (its contributions in term order),
// splitting products with more than kMaxFac factors into chained records.
void emit_entry(const std::vector<Contribution>& cs, std::vector<Rec>& out) {
  for (size_t c = 0; c < cs.size(); ++c) {
    const Contribution& C = cs[c];
    const bool last_contrib = (c + 1 == cs.size());
    size_t pos = 0;
    bool first_chunk = true;
    do {
      Rec r;
      std::memset(&r, 0, sizeof(r));
      r.cre = first_chunk ? C.cre : 0.0;
      r.cim = first_chunk ? C.cim : 0.0;
      r.dest = (uint16_t)C.dest;
      const size_t take = std::min<size_t>(kMaxFac, C.fac.size() - pos);
      r.nf = (uint8_t)take;
      for (size_t q = 0; q < take; ++q) r.fac[q] = (uint16_t)C.fac[pos + q];
      pos += take;
      uint8_t flags = 0;
      if (!first_chunk) flags |= kRecContIn;
      if (pos < C.fac.size()) {
        flags |= kRecContOut;
      } else if (last_contrib) {
        flags |= kRecLast;
      }
      r.flags = flags;
      out.push_back(r);
      first_chunk = false;
    } while (pos < C.fac.size());
  }
}

// Longest-processing-time assignment of entries to the 32 lanes; records
// laid out lane by lane, entries of a lane in increasing entry order.
void schedule(const std::vector<std::vector<Contribution>>& entries,
              std::vector<Rec>& recs, int32_t lane_begin[kWarp + 1]) {
  const int ne = (int)entries.size();
  std::vector<long> cost(ne, 0);
  for (int e = 0; e < ne; ++e)
    for (const auto& c : entries[e]) cost[e] += 2 + (long)c.fac.size();
  std::vector<int> order(ne);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<long> load(kWarp, 0);
  std::vector<std::vector<int>> lane_entries(kWarp);
  for (int e : order) {
    if (entries[e].empty()) continue;
    int best = 0;
    for (int l = 1; l < kWarp; ++l)
      if (load[l] < load[best]) best = l;
    load[best] += cost[e];
    lane_entries[best].push_back(e);
  }
  recs.clear();
  for (int l = 0; l < kWarp; ++l) {
    lane_begin[l] = (int32_t)recs.size();
    std::sort(lane_entries[l].begin(), lane_entries[l].end());
    for (int e : lane_entries[l]) emit_entry(entries[e], recs);
  }
  lane_begin[kWarp] = (int32_t)recs.size();
}

}  // namespace

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

int build_plan(const phc_system* sys, const phc_homotopy* hom, HostPlan* out) {
  int st = validate_system(sys);
  if (st != PHC_OK) return st;
  if (hom == nullptr || hom->b == nullptr || hom->patch == nullptr) return PHC_ERR_INVALID_INPUT;
  const int n = sys->n, N = n + 1;
  if (N > kMaxN) return PHC_ERR_UNSUPPORTED;
  int maxexp = 0;
  for (size_t q = 0; q < (size_t)sys->nterms * N; ++q) maxexp = std::max(maxexp, sys->hexps[q]);
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

  // contributions per entry, in term order (eval_terms, src/sparse.f90:259-278)
  std::vector<std::vector<Contribution>> fent(n), jent((size_t)n * S);
  for (int i = 0; i < n; ++i) {
    for (int k = sys->first[i]; k < sys->first[i + 1]; ++k) {
      const int* e = sys->hexps + (size_t)k * N;
      const double cre = sys->coefs[2 * k], cim = sys->coefs[2 * k + 1];
      Contribution v;
      v.cre = cre;
      v.cim = cim;
      v.dest = i;
      for (int j = 0; j < N; ++j)
        if (e[j] > 0) v.fac.push_back(e[j] * N + j);
      fent[i].push_back(v);
      for (int j = 0; j < N; ++j) {
        if (e[j] <= 0) continue;
        Contribution d;
        d.cre = (double)e[j] * cre;
        d.cim = (double)e[j] * cim;
        d.dest = i * S + j;
        if (e[j] > 1) d.fac.push_back((e[j] - 1) * N + j);
        for (int l = 0; l < N; ++l)
          if (l != j && e[l] > 0) d.fac.push_back(e[l] * N + l);
        jent[(size_t)i * S + j].push_back(d);
      }
    }
  }
  std::vector<Rec> rf, rj;
  schedule(fent, rf, H.lane_f);
  schedule(jent, rj, H.lane_j);
  H.nrec_f = (int32_t)rf.size();
  H.nrec_j = (int32_t)rj.size();
  const size_t bytes = sizeof(PlanHeader) + (rf.size() + rj.size()) * sizeof(Rec);
  H.total_bytes = (int32_t)bytes;

  out->bytes.resize(bytes);
  std::memcpy(out->bytes.data(), &H, sizeof(H));
  if (!rf.empty()) std::memcpy(out->bytes.data() + sizeof(H), rf.data(), rf.size() * sizeof(Rec));
  if (!rj.empty())
    std::memcpy(out->bytes.data() + sizeof(H) + rf.size() * sizeof(Rec), rj.data(),
                rj.size() * sizeof(Rec));
  out->n = n;
  out->N = N;
  out->S = S;
  out->maxexp = maxexp;
  out->pw_size = pw_size;
  out->nstart = radix;
  out->nrec = H.nrec_f + H.nrec_j;
  return PHC_OK;
}

}  // namespace phc
