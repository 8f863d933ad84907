// mesh_io.cpp -- fixture files: the reference's text format and a binary form.
//
// Text (the reference's): Mesh<Float>(file) in include/util/mesh.hpp:51-80
// reads `ndims solvedim`, the extents (fastest first), then ds, dl, d, du, dw,
// x and u, each prod(dims) values parsed at Float's own precision.  Mesh<double>
// takes u from the line after x (the FP64 solution); Mesh<float> skips that
// line and takes u from the next one (the FP32 solution).  The files are what
// test/gen_testcases.py:50-79 writes: one array per line.  Here the parse is
// strtod / strtof in the "C" locale on the same tokens, which is what the
// stream extraction does, so the values are the reference's bit for bit.
//
// Binary (this library's): a 24 + 4 ndims byte header padded to 8 bytes, then
// the arrays at one precision -- see pentadsolver_mesh.h.
#include <cctype>
#include <clocale>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <locale.h>
#include <string>
#include <vector>

#include "pentad_common.hpp"
#include "pentadsolver_mesh.h"

namespace {

constexpr char kMagic[8] = {'P', 'E', 'N', 'T', 'A', 'F', 'X', '1'};

struct Header {
  int ndims = 0, solvedim = 0, format = PENTADSOLVER_FIXTURE_TEXT;
  int dims[PENTAD_MAXDIM] = {};
  bool has_u = false;
  long long count = 0;       // prod(dims)
  size_t data_offset = 0;    // binary: first array byte; text: first value char
};

void complain(const char *path, const char *what) {
  std::fprintf(stderr, "[penta] fixture %s: %s\n", path ? path : "(null)", what);
}

bool read_file(const char *path, std::string &out) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long size = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (size < 0) {
    std::fclose(f);
    return false;
  }
  out.resize(static_cast<size_t>(size));
  const size_t got = size ? std::fread(&out[0], 1, out.size(), f) : 0;
  std::fclose(f);
  return got == out.size();
}

locale_t c_locale() {
  static locale_t loc = newlocale(LC_ALL_MASK, "C", static_cast<locale_t>(0));
  return loc;
}

// One integer token at p (skipping whitespace); false when none.
bool next_int(const char *&p, const char *end, long long &v) {
  while (p < end && std::isspace(static_cast<unsigned char>(*p))) ++p;
  if (p >= end) return false;
  char *stop = nullptr;
  v = strtoll_l(p, &stop, 10, c_locale());
  if (stop == p || stop > end) return false;
  p = stop;
  return true;
}

bool check_dims(Header &h) {
  if (h.ndims < 1 || h.ndims > PENTAD_MAXDIM || h.solvedim < 0 || h.solvedim >= h.ndims)
    return false;
  h.count = 1;
  for (int k = 0; k < h.ndims; ++k) {
    if (h.dims[k] < 1) return false;
    h.count *= h.dims[k];
    if (h.count > (1LL << 40)) return false;
  }
  return true;
}

bool parse_header(const std::string &buf, Header &h) {
  if (buf.size() >= 24 && std::memcmp(buf.data(), kMagic, 8) == 0) {
    uint32_t w[4];
    std::memcpy(w, buf.data() + 8, sizeof(w));
    if (w[0] != 8 && w[0] != 4) return false;
    if (w[1] < 1 || w[1] > PENTAD_MAXDIM) return false;
    h.format = static_cast<int>(w[0]);
    h.ndims = static_cast<int>(w[1]);
    h.solvedim = static_cast<int>(w[2]);
    h.has_u = w[3] != 0;
    const size_t head = 24 + 4 * static_cast<size_t>(h.ndims);
    if (buf.size() < head) return false;
    for (int k = 0; k < h.ndims; ++k) {
      uint32_t e;
      std::memcpy(&e, buf.data() + 24 + 4 * k, 4);
      if (e > 0x7fffffffu) return false;
      h.dims[k] = static_cast<int>(e);
    }
    if (!check_dims(h)) return false;
    h.data_offset = (head + 7) & ~static_cast<size_t>(7);
    const size_t arrays = h.has_u ? 7 : 6;
    return buf.size() >= h.data_offset + arrays * h.count * static_cast<size_t>(h.format);
  }
  const char *p = buf.data(), *end = buf.data() + buf.size();
  long long nd = 0, sd = 0;
  if (!next_int(p, end, nd) || !next_int(p, end, sd)) return false;
  if (nd < 1 || nd > PENTAD_MAXDIM) return false;
  h.ndims = static_cast<int>(nd);
  h.solvedim = static_cast<int>(sd);
  for (int k = 0; k < h.ndims; ++k) {
    long long e = 0;
    if (!next_int(p, end, e) || e < 1 || e > 0x7fffffff) return false;
    h.dims[k] = static_cast<int>(e);
  }
  h.format = PENTADSOLVER_FIXTURE_TEXT;
  h.has_u = true;
  h.data_offset = static_cast<size_t>(p - buf.data());
  return check_dims(h);
}

template <typename F> F parse_value(const char *p, char **stop);
template <> double parse_value<double>(const char *p, char **stop) {
  return strtod_l(p, stop, c_locale());
}
template <> float parse_value<float>(const char *p, char **stop) {
  return strtof_l(p, stop, c_locale());
}

// n values at F's precision; false when the text runs out or a token is not a
// number.  A token is accepted as the stream extraction accepts it: only
// digits, signs, '.', 'e' and 'E' (no "inf", "nan" or hex), and a value that
// overflows F is an error (the extraction fails there too).
template <typename F>
bool parse_array(const char *&p, const char *end, long long n, F *out) {
  for (long long i = 0; i < n; ++i) {
    while (p < end && std::isspace(static_cast<unsigned char>(*p))) ++p;
    if (p >= end) return false;
    const char *tok = p;
    while (tok < end && !std::isspace(static_cast<unsigned char>(*tok))) {
      const char c = *tok;
      if (!((c >= '0' && c <= '9') || c == '+' || c == '-' || c == '.' || c == 'e' ||
            c == 'E'))
        return false;
      ++tok;
    }
    char *stop = nullptr;
    const F v = parse_value<F>(p, &stop);
    if (stop != tok || !std::isfinite(v)) return false;
    if (out) out[i] = v;
    p = stop;
  }
  return true;
}

template <typename F>
pentadStatus_t fixture_read(const char *path, F *ds, F *dl, F *d, F *du, F *dw, F *x, F *u) {
  if (!path || !ds || !dl || !d || !du || !dw || !x) return PENTAD_STATUS_INVALID_VALUE;
  if (c_locale() == static_cast<locale_t>(0)) return PENTAD_STATUS_INTERNAL_ERROR;
  std::string buf;
  if (!read_file(path, buf)) {
    complain(path, "cannot be read");
    return PENTAD_STATUS_INVALID_VALUE;
  }
  Header h;
  if (!parse_header(buf, h)) {
    complain(path, "malformed header or truncated arrays");
    return PENTAD_STATUS_INVALID_VALUE;
  }
  F *const arrays[7] = {ds, dl, d, du, dw, x, u};
  if (h.format != PENTADSOLVER_FIXTURE_TEXT) {
    if (h.format != static_cast<int>(sizeof(F))) {
      complain(path, "binary file holds the other precision");
      return PENTAD_STATUS_INVALID_VALUE;
    }
    if (u && !h.has_u) {
      complain(path, "binary file holds no solution (u)");
      return PENTAD_STATUS_INVALID_VALUE;
    }
    const size_t bytes = static_cast<size_t>(h.count) * sizeof(F);
    for (int a = 0; a < 7; ++a)
      if (arrays[a]) std::memcpy(arrays[a], buf.data() + h.data_offset + a * bytes, bytes);
    return PENTAD_STATUS_SUCCESS;
  }
  // Text: parse into a staging copy first so a malformed file writes nothing.
  std::vector<F> stage(static_cast<size_t>(h.count) * (u ? 7 : 6));
  const char *p = buf.data() + h.data_offset, *end = buf.data() + buf.size();
  for (int a = 0; a < 6; ++a)
    if (!parse_array<F>(p, end, h.count, stage.data() + a * h.count)) {
      complain(path, "an array is short or not numeric");
      return PENTAD_STATUS_INVALID_VALUE;
    }
  if (u) {
    if (sizeof(F) == 4) {
      // Mesh<float>: skip whitespace, then the rest of that line (the FP64 u)
      while (p < end && std::isspace(static_cast<unsigned char>(*p))) ++p;
      while (p < end && *p != '\n') ++p;
    }
    if (!parse_array<F>(p, end, h.count, stage.data() + 6 * h.count)) {
      complain(path, "the solution (u) is short or not numeric");
      return PENTAD_STATUS_INVALID_VALUE;
    }
  }
  for (int a = 0; a < (u ? 7 : 6); ++a)
    std::memcpy(arrays[a], stage.data() + a * h.count, sizeof(F) * h.count);
  return PENTAD_STATUS_SUCCESS;
}

template <typename F>
bool write_text_array(FILE *f, const F *a, long long n, bool as_float) {
  for (long long i = 0; i < n; ++i) {
    const int r = as_float ? std::fprintf(f, i ? " %.9g" : "%.9g", static_cast<double>(
                                                                         static_cast<float>(a[i])))
                           : std::fprintf(f, i ? " %.17g" : "%.17g", static_cast<double>(a[i]));
    if (r < 0) return false;
  }
  return std::fputc('\n', f) != EOF;
}

template <typename F>
pentadStatus_t fixture_write(const char *path, int format, int ndims, int solvedim,
                             const int *dims, const F *ds, const F *dl, const F *d,
                             const F *du, const F *dw, const F *x, const F *u) {
  if (!path || !dims || !ds || !dl || !d || !du || !dw || !x) return PENTAD_STATUS_INVALID_VALUE;
  if (format != PENTADSOLVER_FIXTURE_TEXT && format != static_cast<int>(sizeof(F)))
    return PENTAD_STATUS_INVALID_VALUE;
  if (c_locale() == static_cast<locale_t>(0)) return PENTAD_STATUS_INTERNAL_ERROR;
  Header h;
  h.ndims = ndims;
  h.solvedim = solvedim;
  if (ndims < 1 || ndims > PENTAD_MAXDIM) return PENTAD_STATUS_INVALID_VALUE;
  for (int k = 0; k < ndims; ++k) h.dims[k] = dims[k];
  if (!check_dims(h)) return PENTAD_STATUS_INVALID_VALUE;
  FILE *f = std::fopen(path, "wb");
  if (!f) {
    complain(path, "cannot be created");
    return PENTAD_STATUS_INVALID_VALUE;
  }
  const F *const arrays[6] = {ds, dl, d, du, dw, x};
  bool ok = true;
  if (format == PENTADSOLVER_FIXTURE_TEXT) {
    // The C locale for the decimal point, whatever the caller's is.
    locale_t old = uselocale(c_locale());
    ok = std::fprintf(f, "%d %d\n", ndims, solvedim) > 0;
    for (int k = 0; ok && k < ndims; ++k)
      ok = std::fprintf(f, k ? " %d" : "%d", dims[k]) > 0;
    ok = ok && std::fputc('\n', f) != EOF;
    const bool single = sizeof(F) == 4;
    for (int a = 0; ok && a < 6; ++a) ok = write_text_array<F>(f, arrays[a], h.count, single);
    std::vector<F> zeros;
    const F *sol = u;
    if (!sol) {
      zeros.assign(static_cast<size_t>(h.count), F(0));
      sol = zeros.data();
    }
    ok = ok && write_text_array<F>(f, sol, h.count, single);
    ok = ok && write_text_array<F>(f, sol, h.count, true);
    uselocale(old);
  } else {
    uint32_t w[4] = {static_cast<uint32_t>(sizeof(F)), static_cast<uint32_t>(ndims),
                     static_cast<uint32_t>(solvedim), u ? 1u : 0u};
    ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(w, 4, 4, f) == 4;
    for (int k = 0; ok && k < ndims; ++k) {
      const uint32_t e = static_cast<uint32_t>(dims[k]);
      ok = std::fwrite(&e, 4, 1, f) == 1;
    }
    const size_t head = 24 + 4 * static_cast<size_t>(ndims);
    const char pad[8] = {};
    const size_t npad = ((head + 7) & ~static_cast<size_t>(7)) - head;
    ok = ok && (npad == 0 || std::fwrite(pad, 1, npad, f) == npad);
    for (int a = 0; ok && a < 6; ++a)
      ok = std::fwrite(arrays[a], sizeof(F), h.count, f) == static_cast<size_t>(h.count);
    if (ok && u) ok = std::fwrite(u, sizeof(F), h.count, f) == static_cast<size_t>(h.count);
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    complain(path, "write failed");
    return PENTAD_STATUS_EXECUTION_FAILED;
  }
  return PENTAD_STATUS_SUCCESS;
}

}  // namespace

extern "C" PENTAD_API pentadStatus_t pentadsolver_fixture_info(const char *path, int *ndims,
                                                               int *solvedim, int *dims,
                                                               int *format) {
  if (!path || !ndims || !solvedim || !dims || !format) return PENTAD_STATUS_INVALID_VALUE;
  if (c_locale() == static_cast<locale_t>(0)) return PENTAD_STATUS_INTERNAL_ERROR;
  std::string buf;
  if (!read_file(path, buf)) {
    complain(path, "cannot be read");
    return PENTAD_STATUS_INVALID_VALUE;
  }
  Header h;
  if (!parse_header(buf, h)) {
    complain(path, "malformed header or truncated arrays");
    return PENTAD_STATUS_INVALID_VALUE;
  }
  *ndims = h.ndims;
  *solvedim = h.solvedim;
  *format = h.format;
  for (int k = 0; k < h.ndims; ++k) dims[k] = h.dims[k];
  return PENTAD_STATUS_SUCCESS;
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_D_fixture_read(const char *path, double *ds,
                                                                 double *dl, double *d,
                                                                 double *du, double *dw,
                                                                 double *x, double *u) {
  return fixture_read<double>(path, ds, dl, d, du, dw, x, u);
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_S_fixture_read(const char *path, float *ds,
                                                                 float *dl, float *d,
                                                                 float *du, float *dw,
                                                                 float *x, float *u) {
  return fixture_read<float>(path, ds, dl, d, du, dw, x, u);
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_D_fixture_write(
    const char *path, int format, int ndims, int solvedim, const int *dims, const double *ds,
    const double *dl, const double *d, const double *du, const double *dw, const double *x,
    const double *u) {
  return fixture_write<double>(path, format, ndims, solvedim, dims, ds, dl, d, du, dw, x, u);
}

extern "C" PENTAD_API pentadStatus_t pentadsolver_S_fixture_write(
    const char *path, int format, int ndims, int solvedim, const int *dims, const float *ds,
    const float *dl, const float *d, const float *du, const float *dw, const float *x,
    const float *u) {
  return fixture_write<float>(path, format, ndims, solvedim, dims, ds, dl, d, du, dw, x, u);
}
