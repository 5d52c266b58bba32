// phc_wire.cpp -- the compact request format of the serving path.
//
// A request is one sparse system plus, optionally, its solve_options, in
// a byte string that a client can build without this library's structures.
// The terms carry only their nonzero affine exponents as (variable,
// exponent) pairs, so the size grows with the number of nonzero exponents
// rather than with n times the number of terms. Decoding goes through the
// sparse_system builder (phc_sparse_add_equation), so a decoded request
// obeys exactly the reference's rules for add_equation
// (src/sparse.f90:83-141): zero terms dropped, degree from the kept terms,
// homogenizing exponent d_i - |a|.
//
// Layout (little-endian, no padding):
//   char     magic[4]    "PHCR"
//   uint32   version     1
//   int32    n           unknowns = equations
//   int32    nterms      total number of terms
//   uint32   flags       bit 0: solve options follow
//   uint32   reserved    0
//   [phc_solve_options]  if flags bit 0 (the C struct, byte for byte)
//   int32    terms[n]    terms per equation, in equation order
//   per term, equation by equation:
//     float64 re, im     coefficient
//     uint16  nnz        nonzero affine exponents
//     nnz x { uint16 var (0-based, < n), uint16 exp (> 0) }
#include <cstring>
#include <vector>

#include "phc_host.h"

namespace {

constexpr char kMagic[4] = {'P', 'H', 'C', 'R'};
constexpr uint32_t kVersion = 1;
constexpr size_t kHeader = 24;

struct Reader {
  const unsigned char* p;
  int64_t left;
  template <typename T>
  bool get(T* v) {
    if (left < (int64_t)sizeof(T)) return false;
    std::memcpy(v, p, sizeof(T));
    p += sizeof(T);
    left -= (int64_t)sizeof(T);
    return true;
  }
};

template <typename T>
void put(unsigned char*& q, T v) {
  std::memcpy(q, &v, sizeof(T));
  q += sizeof(T);
}

int64_t encoded_size(const phc_system* sys, bool with_opts) {
  const int N = sys->n + 1;
  int64_t bytes = kHeader + (with_opts ? (int64_t)sizeof(phc_solve_options) : 0) +
                  4 * (int64_t)sys->n;
  for (int k = 0; k < sys->nterms; ++k) {
    int nnz = 0;
    for (int j = 0; j < sys->n; ++j) nnz += sys->hexps[(size_t)k * N + j] > 0 ? 1 : 0;
    bytes += 16 + 2 + 4 * (int64_t)nnz;
  }
  return bytes;
}

}  // namespace

using namespace phc;

extern "C" {

int64_t phc_request_size(const phc_system* sys, int32_t with_options) {
  if (validate_system(sys) != PHC_OK) return -1;
  return encoded_size(sys, with_options != 0);
}

int32_t phc_request_encode(const phc_system* sys, const phc_solve_options* opts, void* buf,
                           int64_t cap, int64_t* len) {
  int st = validate_system(sys);
  if (st != PHC_OK) return st;
  if (!buf || !len) return PHC_ERR_INVALID_INPUT;
  const int n = sys->n, N = n + 1;
  for (int k = 0; k < sys->nterms; ++k)
    for (int j = 0; j < n; ++j)
      if (sys->hexps[(size_t)k * N + j] > 0xffff) return PHC_ERR_UNSUPPORTED;
  if (n > 0xffff) return PHC_ERR_UNSUPPORTED;
  const int64_t need = encoded_size(sys, opts != nullptr);
  *len = need;
  if (cap < need) {
    set_last_error("request buffer too small");
    return PHC_ERR_INVALID_INPUT;
  }
  unsigned char* q = static_cast<unsigned char*>(buf);
  std::memcpy(q, kMagic, 4);
  q += 4;
  put<uint32_t>(q, kVersion);
  put<int32_t>(q, n);
  put<int32_t>(q, sys->nterms);
  put<uint32_t>(q, opts ? 1u : 0u);
  put<uint32_t>(q, 0u);
  if (opts) {
    std::memcpy(q, opts, sizeof(phc_solve_options));
    q += sizeof(phc_solve_options);
  }
  for (int i = 0; i < n; ++i) put<int32_t>(q, sys->first[i + 1] - sys->first[i]);
  for (int k = 0; k < sys->nterms; ++k) {
    put<double>(q, sys->coefs[2 * k]);
    put<double>(q, sys->coefs[2 * k + 1]);
    const int32_t* e = sys->hexps + (size_t)k * N;
    uint16_t nnz = 0;
    for (int j = 0; j < n; ++j) nnz += e[j] > 0 ? 1 : 0;
    put<uint16_t>(q, nnz);
    for (int j = 0; j < n; ++j) {
      if (e[j] <= 0) continue;
      put<uint16_t>(q, (uint16_t)j);
      put<uint16_t>(q, (uint16_t)e[j]);
    }
  }
  return PHC_OK;
}

int32_t phc_request_decode(const void* buf, int64_t len, phc_sparse* builder,
                           phc_solve_options* opts) {
  if (!buf || !builder || len < (int64_t)kHeader) return PHC_ERR_INVALID_INPUT;
  Reader r{static_cast<const unsigned char*>(buf), len};
  char magic[4];
  std::memcpy(magic, r.p, 4);
  r.p += 4;
  r.left -= 4;
  uint32_t version = 0, flags = 0, reserved = 0;
  int32_t n = 0, nterms = 0;
  if (std::memcmp(magic, kMagic, 4) != 0 || !r.get(&version) || version != kVersion ||
      !r.get(&n) || !r.get(&nterms) || !r.get(&flags) || !r.get(&reserved) || n < 1 ||
      n > 0xffff || nterms < 0) {
    set_last_error("not a request of this format");
    return PHC_ERR_INVALID_INPUT;
  }
  phc_solve_options o = solve_defaults();
  if (flags & 1u) {
    if (r.left < (int64_t)sizeof(phc_solve_options)) return PHC_ERR_INVALID_INPUT;
    std::memcpy(&o, r.p, sizeof(phc_solve_options));
    r.p += sizeof(phc_solve_options);
    r.left -= (int64_t)sizeof(phc_solve_options);
  }
  std::vector<int32_t> counts(n);
  int64_t total = 0;
  for (int i = 0; i < n; ++i) {
    if (!r.get(&counts[i]) || counts[i] < 0) return PHC_ERR_INVALID_INPUT;
    total += counts[i];
  }
  if (total != nterms) {
    set_last_error("term counts do not add up");
    return PHC_ERR_INVALID_INPUT;
  }
  int st = phc_sparse_init(builder, n);
  if (st != PHC_OK) return st;
  std::vector<double> coefs;
  std::vector<int32_t> exps;
  for (int i = 0; i < n; ++i) {
    const int nt = counts[i];
    coefs.assign(2 * (size_t)nt, 0.0);
    exps.assign((size_t)nt * n, 0);
    for (int k = 0; k < nt; ++k) {
      uint16_t nnz = 0;
      if (!r.get(&coefs[2 * k]) || !r.get(&coefs[2 * k + 1]) || !r.get(&nnz))
        return PHC_ERR_INVALID_INPUT;
      for (int q = 0; q < nnz; ++q) {
        uint16_t var = 0, e = 0;
        if (!r.get(&var) || !r.get(&e) || var >= n || e == 0) {
          set_last_error("bad (variable, exponent) pair");
          return PHC_ERR_INVALID_INPUT;
        }
        exps[(size_t)k * n + var] += e;
      }
    }
    st = phc_sparse_add_equation(builder, nt, coefs.data(), n, nt, exps.data());
    if (st != PHC_OK) return st;
  }
  if (r.left != 0) {
    set_last_error("trailing bytes after the last term");
    return PHC_ERR_INVALID_INPUT;
  }
  if (opts) *opts = o;
  return PHC_OK;
}

int32_t phc_server_submit_request(phc_server* srv, const void* buf, int64_t len,
                                  uint64_t* ticket) {
  if (!srv || !ticket) return PHC_ERR_BAD_HANDLE;
  phc_sparse* b = phc_sparse_create();
  if (!b) return PHC_ERR_OOM;
  phc_solve_options o;
  int st = phc_request_decode(buf, len, b, &o);
  if (st == PHC_OK) {
    phc_system sys;
    st = phc_sparse_table(b, &sys);
    if (st == PHC_OK) st = phc_server_submit(srv, &sys, &o, ticket);  // copies the table
  }
  phc_sparse_destroy(b);
  return st;
}

}  // extern "C"
