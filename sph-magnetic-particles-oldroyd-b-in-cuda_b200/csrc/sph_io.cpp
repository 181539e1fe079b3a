// sph_io.cpp -- the reference's text output files (micro / walls / colloids / gradv /
// macro), byte-identical to its fprintf output, formatted on all host cores.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "sph_io.h"

namespace {

// Unsigned decimal, no padding.  Returns the number of characters.
inline int put_u64(uint64_t v, char* out) {
  char tmp[24];
  int n = 0;
  do {
    tmp[n++] = char('0' + v % 10);
    v /= 10;
  } while (v);
  for (int k = 0; k < n; ++k) out[k] = tmp[n - 1 - k];
  return n;
}

inline int put_int(int v, char* out) {
  if (v < 0) {
    out[0] = '-';
    return 1 + put_u64((uint64_t)(-(int64_t)v), out + 1);
  }
  return put_u64((uint64_t)v, out);
}

// printf("%.8f"): the exact value of the double, x = m * 2^e, scaled by 10^8 and rounded
// to the nearest integer, ties to even (glibc rounds the exact binary value in the
// default rounding mode).  m * 10^8 < 2^80 fits in 128 bits; the shift keeps the
// remainder for the rounding decision.  |x| >= 9e10 (the scaled value would pass 2^63),
// infinities and NaNs go through snprintf itself.
int fixed8(double x, char* out) {
  if (!(std::fabs(x) < 9.0e10)) return std::snprintf(out, 330, "%.8f", x);
  uint64_t bits;
  std::memcpy(&bits, &x, sizeof(bits));
  const bool neg = (bits >> 63) != 0;
  const int bexp = (int)((bits >> 52) & 0x7ff);
  uint64_t mant = bits & ((1ull << 52) - 1);
  int e;
  if (bexp == 0) {
    e = -1074;
  } else {
    mant |= 1ull << 52;
    e = bexp - 1075;
  }
  const unsigned __int128 v = (unsigned __int128)mant * 100000000u;
  unsigned __int128 q;
  if (e >= 0) {
    q = v << e;  // |x| < 9e10 bounds this below 9e18
  } else if (-e >= 128) {
    q = 0;  // v < 2^80 is below half of 2^-e
  } else {
    const int s = -e;
    q = v >> s;
    const unsigned __int128 rem = v - (q << s);
    const unsigned __int128 half = (unsigned __int128)1 << (s - 1);
    if (rem > half || (rem == half && (q & 1))) ++q;
  }
  const uint64_t Q = (uint64_t)q;
  char* p = out;
  if (neg) *p++ = '-';
  p += put_u64(Q / 100000000u, p);
  *p++ = '.';
  uint64_t f = Q % 100000000u;
  for (int k = 7; k >= 0; --k) {
    p[k] = char('0' + f % 10);
    f /= 10;
  }
  p += 8;
  return (int)(p - out);
}

// One output column: a double array (printed with "%.8f"), or the int array printed with
// "%d"; with g9, the double array rounded to float and printed with "%.9g", the shortest
// form that reads back as the same float for every value.
struct Col {
  const double* d;
  const int* i;
  bool g9 = false;
};

inline int put_col(const Col& c, int64_t r, char* p) {
  if (c.g9) {
    const double v = c.d ? (double)(float)c.d[r] : (double)(float)c.i[r];
    return std::snprintf(p, 32, "%.9g", v);
  }
  return c.d ? fixed8(c.d[r], p) : put_int(c.i[r], p);
}

// Writes rows "idx c0 c1 ... <end>" for idx = 0..n-1 (without the index, "c0 c1 ... <end>"),
// formatted in parallel chunks.
sph_status write_rows(const char* path, int n, const std::vector<Col>& cols, const char* end,
                      bool index = true) {
  FILE* f = std::fopen(path, "w");
  if (!f) return SPH_ERR_IO;
  const int64_t chunk = 32768;
  const int64_t nchunks = (n + chunk - 1) / chunk;
  unsigned hw = std::thread::hardware_concurrency();
  const int nthreads = (int)std::max<int64_t>(1, std::min<int64_t>(hw ? hw : 1, nchunks));
  const size_t endlen = std::strlen(end);
  // typical row (values below 1e10) and the worst case (snprintf of a huge value)
  const size_t row_typ = 16 + cols.size() * 24 + endlen;
  const size_t row_max = 16 + cols.size() * 330 + endlen;
  bool ok = true;
  // rounds of nthreads chunks: format in parallel, write in order
  std::vector<std::string> buf(nthreads);
  for (int64_t c0 = 0; c0 < nchunks && ok; c0 += nthreads) {
    const int nt = (int)std::min<int64_t>(nthreads, nchunks - c0);
    auto work = [&](int t) {
      const int64_t a = (c0 + t) * chunk, b = std::min<int64_t>(n, a + chunk);
      std::string& s = buf[t];
      s.resize((size_t)(b - a) * row_typ + row_max);
      size_t off = 0;
      for (int64_t r = a; r < b; ++r) {
        if (off + row_max > s.size()) s.resize(std::max(2 * s.size(), off + row_max));
        char* p = &s[off];
        if (index) p += put_int((int)r, p);
        bool first = !index;
        for (const Col& c : cols) {
          if (!first) *p++ = ' ';
          first = false;
          p += put_col(c, r, p);
        }
        std::memcpy(p, end, endlen);
        p += endlen;
        off = (size_t)(p - &s[0]);
      }
      s.resize(off);
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& t : th) t.join();
    for (int t = 0; t < nt && ok; ++t)
      ok = std::fwrite(buf[t].data(), 1, buf[t].size(), f) == buf[t].size();
  }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? SPH_OK : SPH_ERR_IO;
}

bool dim_ok(int dim) { return dim == 2 || dim == 3; }

}  // namespace

extern "C" {

int sph_format_fixed8(double x, char* buf) {
  const int n = fixed8(x, buf);
  buf[n] = '\0';
  return n;
}

sph_status sph_write_micro(const char* path, int dim, int n, const double* x, const double* y,
                           const double* z, const double* vx, const double* vy,
                           const double* vz, const double* mass, const double* dens,
                           const double* press, const int* type, const double* cxx,
                           const double* cxy, const double* cyy, const double* cxz,
                           const double* cyz, const double* czz) {
  if (!path || !dim_ok(dim) || n < 0) return SPH_ERR_STATE;
  const std::vector<Col> c =
      dim == 2 ? std::vector<Col>{{x, 0}, {y, 0}, {vx, 0}, {vy, 0}, {mass, 0}, {dens, 0},
                                  {press, 0}, {0, type}, {cxx, 0}, {cxy, 0}, {cyy, 0}}
               : std::vector<Col>{{x, 0},     {y, 0},    {z, 0},   {vx, 0},  {vy, 0},
                                  {vz, 0},    {mass, 0}, {dens, 0}, {press, 0}, {0, type},
                                  {cxx, 0},   {cxy, 0},  {cyy, 0}, {cxz, 0}, {cyz, 0},
                                  {czz, 0}};
  for (const Col& k : c)
    if (!k.d && !k.i) return SPH_ERR_STATE;
  return write_rows(path, n, c, dim == 2 ? " \n" : "\n");
}

sph_status sph_write_walls(const char* path, int dim, int nwalls, const double* fx,
                           const double* fy, const double* fz) {
  if (!path || !dim_ok(dim) || nwalls < 0 || !fx || !fy || (dim == 3 && !fz))
    return SPH_ERR_STATE;
  std::vector<Col> c = {{fx, 0}, {fy, 0}};
  if (dim == 3) c.push_back({fz, 0});
  return write_rows(path, nwalls, c, "\n");
}

sph_status sph_write_colloids(const char* path, int dim, int n, const double* const* f) {
  if (!path || !dim_ok(dim) || n < 0 || !f) return SPH_ERR_STATE;
  // 3D order: x y z vx vy vz ox oy oz fx fy fz tx ty tz
  const int pick2[] = {0, 1, 3, 4, 8, 9, 10, 14};
  std::vector<Col> c;
  if (dim == 2)
    for (int k : pick2) c.push_back({f[k], 0});
  else
    for (int k = 0; k < 15; ++k) c.push_back({f[k], 0});
  for (const Col& k : c)
    if (!k.d) return SPH_ERR_STATE;
  return write_rows(path, n, c, "\n");
}

sph_status sph_write_gradv(const char* path, int dim, int n, const double* x, const double* y,
                           const double* z, const double* const* g) {
  if (!path || !dim_ok(dim) || n < 0 || !g) return SPH_ERR_STATE;
  std::vector<Col> c{{x, 0}, {y, 0}};
  if (dim == 2) {
    for (int k : {0, 1, 3, 4}) c.push_back({g[k], 0});
  } else {
    c.push_back({z, 0});
    for (int k = 0; k < 9; ++k) c.push_back({g[k], 0});
  }
  for (const Col& k : c)
    if (!k.d) return SPH_ERR_STATE;
  return write_rows(path, n, c, "\n");
}

sph_status sph_write_restart(const char* path, int dim, int n, const double* x, const double* y,
                             const double* z, const double* vx, const double* vy,
                             const double* vz, const double* mass, const int* type,
                             const double* cxx, const double* cxy, const double* cyy,
                             const double* cxz, const double* cyz, const double* czz) {
  if (!path || !dim_ok(dim) || n < 0) return SPH_ERR_STATE;
  auto g = [](const double* d) { return Col{d, nullptr, true}; };
  const Col t{nullptr, type, true};
  const std::vector<Col> c =
      dim == 2 ? std::vector<Col>{g(x), g(y), g(vx), g(vy), g(mass), t, g(cxx), g(cxy), g(cyy)}
               : std::vector<Col>{g(x),   g(y),   g(z),   g(vx),  g(vy),  g(vz),  g(mass),
                                  t,      g(cxx), g(cxy), g(cyy), g(cxz), g(cyz), g(czz)};
  for (const Col& k : c)
    if (!k.d && !k.i) return SPH_ERR_STATE;
  return write_rows(path, n, c, "\n", false);
}

sph_status sph_append_macro(const char* path, int step, double kin_energy) {
  if (!path) return SPH_ERR_STATE;
  FILE* f = std::fopen(path, step == 0 ? "w" : "a");
  if (!f) return SPH_ERR_IO;
  const bool ok = std::fprintf(f, "%d %f\n", step, kin_energy) > 0;
  return (std::fclose(f) == 0 && ok) ? SPH_OK : SPH_ERR_IO;
}

}  // extern "C"
