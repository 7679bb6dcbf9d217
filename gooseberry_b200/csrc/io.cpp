// io.cpp -- CSR and grid text files: the reference's readers and writers
// (src/io.c:145-239 __read_grid, 369-498 __read_csr, 1195-1229 __write_grid,
// 1233-1275 __write_csr) with the same format rules, parsed by all host
// threads, plus gb_csr_read, which parses straight into a device matrix.
//
// Format rules kept from the reference:
//  - lines end at '\n'; the newline that ends the file opens no extra line;
//  - a line whose first character is one of  # % ' " /  is a comment;
//  - CSR: every other line is a row of "column value" pairs read with
//    strtoull / strtod until a value fails to parse; a blank line is an empty
//    row; columns are 1-based unless a 0 appears (the smallest column seen,
//    capped at 1, is subtracted); ncols = largest - smallest + 1;
//  - grid: every non-comment line is a row of values; the first line fixes the
//    column count (a leading blank line leaves it open), a later line with no
//    values or a different count is an error;
//  - writers print values with %g and CSR columns 1-based, one row per line.
//
// The file is read into memory once; newlines become terminators so strtod
// never runs into the next line, lines are found by parallel chunk scans, and
// rows are parsed by contiguous line ranges per thread and concatenated in
// order, so the arrays are exactly the sequential reader's.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <charconv>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <condition_variable>
#include <memory>
#include <mutex>
#include <new>
#include <string>

#include <sys/stat.h>
#include <unistd.h>
#include <thread>
#include <vector>

#include "gb_internal.h"

namespace gb {
namespace {

bool is_comment(char c) {
  return c == '#' || c == '%' || c == '\'' || c == '"' || c == '/';
}

unsigned n_threads() {
  return std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
}

// body(t) for t in [0, nt), on nt threads (the caller's among them).  A
// thread that cannot be started runs its share inline instead: nothing
// throws through the C interface.
template <class F>
void parallel_for(unsigned nt, F && body) {
  std::vector<std::thread> th;
  unsigned t = 1;
  try {
    th.reserve(nt);
    for (; t < nt; ++t) th.emplace_back(body, t);
  } catch (...) {
    for (unsigned u = t; u < nt; ++u) body(u);
  }
  body(0u);
  for (auto & x : th) x.join();
}

int open_error(const char * path, const char * mode) {
  if (errno == ENOENT || errno == ENOTDIR) {
    set_error("file not found '%s'", path);
    return GOOSEBERRY_ERROR_FILENOTFOUND;
  }
  if (errno == EACCES) {
    set_error("permission denied '%s'", path);
    return GOOSEBERRY_ERROR_PERMISSIONDENIED;
  }
  set_error("cannot open '%s' (%s) for %s", path, std::strerror(errno),
      mode[0] == 'r' ? "reading" : "writing");
  return GOOSEBERRY_ERROR_UNKNOWN;
}

// The whole file, newlines replaced by '\0', and the start of every line.
struct Lines {
  std::unique_ptr<char[]> buf;  // not zero-filled: every byte is read from the file
  std::vector<size_t> start;    // line i spans buf[start[i]] .. its '\0'
};

int read_lines(const char * path, Lines & L) {
  GB_CHECK_INPUT(path != nullptr, "file name is NULL");
  FILE * f = std::fopen(path, "rb");
  if (!f) return open_error(path, "r");
  struct stat st;
  const bool regular = fstat(fileno(f), &st) == 0 && S_ISREG(st.st_mode) && st.st_size > 0;
  size_t cap = regular ? static_cast<size_t>(st.st_size) : (1u << 20);
  L.buf.reset(new char[cap + 1]);
  size_t got = 0;
  if (regular) {
    // a regular file of known size: every thread reads its own byte range
    // (the copy out of the page cache is the slow part of a single read)
    const unsigned nr = static_cast<unsigned>(std::min<size_t>(n_threads(),
        std::max<size_t>(cap >> 24, 1)));
    std::vector<size_t> part(nr, 0);
    const int fd = fileno(f);
    parallel_for(nr, [&](unsigned t) {
      const size_t a = cap * t / nr, b = cap * (t + 1) / nr;
      size_t done = 0;
      while (a + done < b) {
        const ssize_t r = pread(fd, L.buf.get() + a + done, b - a - done,
            static_cast<off_t>(a + done));
        if (r <= 0) break;
        done += static_cast<size_t>(r);
      }
      part[t] = done;
    });
    // contiguous prefix that was read; the loop below reads whatever is left
    for (unsigned t = 0; t < nr; ++t) {
      got += part[t];
      if (part[t] != cap * (t + 1) / nr - cap * t / nr) break;
    }
    std::fseek(f, static_cast<long>(got), SEEK_SET);
  }
  for (;;) {  // the size is a hint: read to the end whatever it is
    got += std::fread(L.buf.get() + got, 1, cap - got, f);
    if (got < cap || std::feof(f)) break;
    int c = std::fgetc(f);
    if (c == EOF) break;
    std::unique_ptr<char[]> bigger(new char[2 * cap + 1]);
    std::memcpy(bigger.get(), L.buf.get(), got);
    bigger[got++] = static_cast<char>(c);
    L.buf = std::move(bigger);
    cap *= 2;
  }
  const bool bad = std::ferror(f) != 0;
  std::fclose(f);
  if (bad) {
    set_error("read error on '%s'", path);
    return GOOSEBERRY_ERROR_READ;
  }
  const size_t n = got;
  char * buf = L.buf.get();
  buf[n] = '\0';
  // newline positions, chunk-parallel, in order
  const unsigned nt = n_threads();
  std::vector<std::vector<size_t>> nl(nt);
  parallel_for(nt, [&](unsigned t) {
    const size_t a = n * t / nt, b = n * (t + 1) / nt;
    const char * p = buf + a;
    const char * const e = buf + b;
    while (p < e) {
      const char * q = static_cast<const char *>(std::memchr(p, '\n', static_cast<size_t>(e - p)));
      if (!q) break;
      nl[t].push_back(static_cast<size_t>(q - buf));
      p = q + 1;
    }
  });
  // line starts, filled by every thread for its own newlines: thread t's
  // first line starts after the last newline any earlier thread found
  std::vector<size_t> first(nt + 1, 0), from(nt, 0);
  size_t prev = 0;
  for (unsigned t = 0; t < nt; ++t) {
    first[t + 1] = first[t] + nl[t].size();
    from[t] = prev;
    if (!nl[t].empty()) prev = nl[t].back() + 1;
  }
  const size_t total = first[nt];
  const bool tail = n > 0 && buf[n - 1] != '\n';  // last line without a newline
  L.start.resize(total + (tail ? 1 : 0));
  parallel_for(nt, [&](unsigned t) {
    size_t k = first[t], p = from[t];
    for (size_t pos : nl[t]) {
      L.start[k++] = p;
      buf[pos] = '\0';
      p = pos + 1;
    }
  });
  if (tail) L.start[total] = prev;
  return GOOSEBERRY_SUCCESS;
}

template <typename T>
struct CsrPart {
  std::vector<uint32_t> count;  // entries per row, in line order
  std::vector<uint32_t> ind;
  std::vector<T> val;
  uint32_t mincol = 1, maxcol = 0;
};

bool is_space(char c) {
  return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f';
}

// strtoull(s, &end, 10) with a fast path for [spaces] digits (no sign, no
// overflow); anything else goes to strtoull itself.
unsigned long long parse_ull(const char * s, char ** end) {
  const char * q = s;
  while (is_space(*q)) ++q;
  unsigned long long v = 0;
  int nd = 0;
  while (*q >= '0' && *q <= '9' && nd < 19) {
    v = v * 10 + static_cast<unsigned>(*q - '0');
    ++q;
    ++nd;
  }
  if (nd == 0 || (*q >= '0' && *q <= '9')) return std::strtoull(s, end, 10);
  *end = const_cast<char *>(q);
  return v;
}

// strtod(s, &end) with a fast path: a plain decimal token ([+-] digits, '.',
// exponent) is converted by std::from_chars, which rounds correctly like
// strtod; hex, inf, nan and anything odd go to strtod itself.
double parse_double(const char * s, char ** end) {
  const char * q = s;
  while (is_space(*q)) ++q;
  const char * t = q;
  bool neg = false;
  if (*t == '+' || *t == '-') {
    neg = *t == '-';
    ++t;
  }
  if (!((*t >= '0' && *t <= '9') || (*t == '.' && t[1] >= '0' && t[1] <= '9')) ||
      (t[0] == '0' && (t[1] == 'x' || t[1] == 'X')))
    return std::strtod(s, end);
  const char * e = t;
  while (*e && !is_space(*e)) ++e;
  double v = 0.0;
  const auto r = std::from_chars(t, e, v, std::chars_format::general);
  if (r.ec != std::errc() || r.ptr != e) return std::strtod(s, end);
  *end = const_cast<char *>(e);
  return neg ? -v : v;
}

// One CSR row: "col val" pairs until a value does not parse (src/io.c:417-437).
template <typename T>
void parse_csr_row(const char * line, CsrPart<T> & p) {
  const char * sptr = line;
  char * eptr = nullptr;
  uint32_t n = 0;
  uint32_t i = static_cast<uint32_t>(parse_ull(sptr, &eptr));
  sptr = eptr;
  double f = parse_double(sptr, &eptr);
  while (eptr != sptr) {
    p.maxcol = std::max(p.maxcol, i);
    p.mincol = std::min(p.mincol, i);
    p.ind.push_back(i);
    p.val.push_back(static_cast<T>(f));
    ++n;
    sptr = eptr;
    i = static_cast<uint32_t>(parse_ull(sptr, &eptr));
    sptr = eptr;
    f = parse_double(sptr, &eptr);
  }
  p.count.push_back(n);
}

template <typename T>
T * malloc_n(size_t n) {
  return static_cast<T *>(std::malloc(sizeof(T) * (n ? n : 1)));
}

// Whitespace-separated tokens of a line: the reference sizes a CSR row as
// this over two (src/io.c:414).
uint32_t count_tokens(const char * s) {
  uint32_t n = 0;
  bool in = false;
  for (; *s; ++s) {
    const bool sp = is_space(*s);
    n += (!sp && !in) ? 1u : 0u;
    in = !sp;
  }
  return n;
}

constexpr uint32_t kCommentLine = 0xffffffffu;

// The common case, in two passes over the lines: every line's token count
// over two sizes its row (one pass, by all threads), then every row is parsed
// straight into the caller's arrays at its offset.  Exact only when each row
// parses into exactly that many pairs, which holds whenever every token reads
// whole as a number; returns false (arrays released) when a row does not, and
// the caller falls back to read_csr_rows.  Columns are stored 1-based minus
// one and shifted back when a 0 column makes the file 0-based (mincol,
// src/io.c:464).
template <typename T, class Alloc, class Release>
bool read_csr_sized(const Lines & L, dim_t * nrows, dim_t * ncols, ind_t ** r_rowptr,
    dim_t ** r_rowind, T ** r_rowval, Alloc && alloc, Release && release, int * rc) {
  const size_t nl = L.start.size();
  const unsigned nt = static_cast<unsigned>(std::min<size_t>(n_threads(),
      std::max<size_t>(nl / 1024, 1)));
  std::vector<uint32_t> pairs(nl);
  std::vector<size_t> rows(nt + 1, 0), ents(nt + 1, 0);
  parallel_for(nt, [&](unsigned t) {
    size_t r = 0, e = 0;
    for (size_t l = nl * t / nt; l < nl * (t + 1) / nt; ++l) {
      const char * line = L.buf.get() + L.start[l];
      if (line[0] != '\0' && is_comment(line[0])) {
        pairs[l] = kCommentLine;
        continue;
      }
      pairs[l] = count_tokens(line) / 2;
      ++r;
      e += pairs[l];
    }
    rows[t + 1] = r;
    ents[t + 1] = e;
  });
  for (unsigned t = 0; t < nt; ++t) {
    rows[t + 1] += rows[t];
    ents[t + 1] += ents[t];
  }
  const size_t n = rows[nt], nnz = ents[nt];
  if (n >= 0xffffffffu || nnz > 0xffffffffu) return false;  // the general path reports it
  ind_t * rowptr = nullptr;
  dim_t * rowind = nullptr;
  T * rowval = nullptr;
  if (!alloc(&rowptr, n + 1) || !alloc(&rowind, nnz) || !alloc(&rowval, nnz)) {
    if (rowptr) release(rowptr);
    if (rowind) release(rowind);
    set_error("out of host memory reading CSR rows");
    *rc = GOOSEBERRY_ERROR_UNKNOWN;
    return true;
  }
  std::vector<uint32_t> lo(nt, 1), hi(nt, 0);
  std::vector<char> bad(nt, 0);
  rowptr[0] = 0;
  parallel_for(nt, [&](unsigned t) {
    size_t r = rows[t], j = ents[t];
    uint32_t mn = 1, mx = 0;
    bool b = false;
    for (size_t l = nl * t / nt; l < nl * (t + 1) / nt && !b; ++l) {
      const uint32_t want = pairs[l];
      if (want == kCommentLine) continue;
      // the loop of src/io.c:423-437, stopped at the row's size
      const char * sptr = L.buf.get() + L.start[l];
      char * eptr = nullptr;
      uint32_t k = 0;
      uint32_t i = static_cast<uint32_t>(parse_ull(sptr, &eptr));
      sptr = eptr;
      double f = parse_double(sptr, &eptr);
      while (eptr != sptr) {
        if (k == want) break;
        mx = std::max(mx, i);
        mn = std::min(mn, i);
        rowind[j + k] = i - 1u;
        rowval[j + k] = static_cast<T>(f);
        ++k;
        sptr = eptr;
        i = static_cast<uint32_t>(parse_ull(sptr, &eptr));
        sptr = eptr;
        f = parse_double(sptr, &eptr);
      }
      b = k != want || eptr != sptr;
      j += want;
      rowptr[++r] = static_cast<ind_t>(j);
    }
    lo[t] = mn;
    hi[t] = mx;
    bad[t] = b;
  });
  uint32_t mincol = 1, maxcol = 0;
  bool exact = true;
  for (unsigned t = 0; t < nt; ++t) {
    mincol = std::min(mincol, lo[t]);
    maxcol = std::max(maxcol, hi[t]);
    exact = exact && !bad[t];
  }
  if (!exact) {
    release(rowptr);
    release(rowind);
    release(rowval);
    return false;
  }
  if (mincol == 0) {  // a 0-based file: undo the 1-based shift
    parallel_for(nt, [&](unsigned t) {
      for (size_t e = nnz * t / nt; e < nnz * (t + 1) / nt; ++e) rowind[e] += 1u;
    });
  }
  *r_rowptr = rowptr;
  *r_rowind = rowind;
  *r_rowval = rowval;
  *nrows = static_cast<dim_t>(n);
  *ncols = maxcol - mincol + 1;
  *rc = GOOSEBERRY_SUCCESS;
  return true;
}

// The general case: rows parsed by all threads into per-thread lists, then
// gathered into caller-owned arrays made by `alloc`.
template <typename T, class Alloc, class Release>
int read_csr_rows(const char * path, const Lines & L, dim_t * nrows, dim_t * ncols,
    ind_t ** r_rowptr, dim_t ** r_rowind, T ** r_rowval, Alloc && alloc, Release && release) {
  const size_t nl = L.start.size();
  const unsigned nt = static_cast<unsigned>(std::min<size_t>(n_threads(),
      std::max<size_t>(nl / 1024, 1)));
  std::vector<CsrPart<T>> part(nt);
  parallel_for(nt, [&](unsigned t) {
    const size_t a = nl * t / nt, b = nl * (t + 1) / nt;
    CsrPart<T> & p = part[t];
    for (size_t l = a; l < b; ++l) {
      const char * line = L.buf.get() + L.start[l];
      if (line[0] != '\0' && is_comment(line[0])) continue;  // blank lines are empty rows
      parse_csr_row(line, p);
    }
  });
  size_t n = 0, nnz = 0;
  uint32_t mincol = 1, maxcol = 0;
  for (auto & p : part) {
    n += p.count.size();
    nnz += p.ind.size();
    mincol = std::min(mincol, p.mincol);
    maxcol = std::max(maxcol, p.maxcol);
  }
  GB_CHECK_INPUT(n < 0xffffffffu && nnz <= 0xffffffffu,
      "'%s' holds %zu rows / %zu entries, beyond 32-bit indices", path, n, nnz);
  ind_t * rowptr = nullptr;
  dim_t * rowind = nullptr;
  T * rowval = nullptr;
  if (!alloc(&rowptr, n + 1) || !alloc(&rowind, nnz) || !alloc(&rowval, nnz)) {
    if (rowptr) release(rowptr);
    if (rowind) release(rowind);
    set_error("out of host memory reading '%s'", path);
    return GOOSEBERRY_ERROR_UNKNOWN;
  }
  std::vector<size_t> row0(nt + 1, 0), ent0(nt + 1, 0);
  for (unsigned t = 0; t < nt; ++t) {
    row0[t + 1] = row0[t] + part[t].count.size();
    ent0[t + 1] = ent0[t] + part[t].ind.size();
  }
  rowptr[0] = 0;
  parallel_for(nt, [&](unsigned t) {
    const CsrPart<T> & p = part[t];
    size_t j = ent0[t];
    for (size_t r = 0; r < p.count.size(); ++r) {
      j += p.count[r];
      rowptr[row0[t] + r + 1] = static_cast<ind_t>(j);
    }
    for (size_t e = 0; e < p.ind.size(); ++e) {
      rowind[ent0[t] + e] = p.ind[e] - mincol;  // mincol is at most 1
      rowval[ent0[t] + e] = p.val[e];
    }
  });
  *r_rowptr = rowptr;
  *r_rowind = rowind;
  *r_rowval = rowval;
  *nrows = static_cast<dim_t>(n);
  *ncols = maxcol - mincol + 1;
  return GOOSEBERRY_SUCCESS;
}

// Parses a CSR file into caller-owned arrays made by `alloc` (and given back
// through `release` when the sized pass cannot be used).
template <typename T, class Alloc, class Release>
int read_csr(const char * path, dim_t * nrows, dim_t * ncols, ind_t ** r_rowptr,
    dim_t ** r_rowind, T ** r_rowval, Alloc && alloc, Release && release) {
  GB_CHECK_INPUT(nrows && ncols && r_rowptr && r_rowind && r_rowval, "NULL output");
  Lines L;
  GB_TRY(read_lines(path, L));
  int rc = GOOSEBERRY_SUCCESS;
  if (read_csr_sized<T>(L, nrows, ncols, r_rowptr, r_rowind, r_rowval, alloc, release, &rc))
    return rc;
  return read_csr_rows<T>(path, L, nrows, ncols, r_rowptr, r_rowind, r_rowval, alloc,
      release);
}

template <typename T>
int read_grid(const char * path, dim_t * r_nrows, dim_t * r_ncols, T ** r_rowval) {
  GB_CHECK_INPUT(r_nrows && r_ncols && r_rowval, "NULL output");
  Lines L;
  GB_TRY(read_lines(path, L));
  const size_t nl = L.start.size();
  // values per line (comments: ~0)
  const size_t kComment = ~size_t(0);
  std::vector<size_t> cnt(nl);
  const unsigned nt = static_cast<unsigned>(std::min<size_t>(n_threads(),
      std::max<size_t>(nl / 256, 1)));
  parallel_for(nt, [&](unsigned t) {
    for (size_t l = nl * t / nt; l < nl * (t + 1) / nt; ++l) {
      const char * line = L.buf.get() + L.start[l];
      if (is_comment(line[0])) {
        cnt[l] = kComment;
        continue;
      }
      size_t j = 0;
      const char * sptr = line;
      char * eptr = nullptr;
      parse_double(sptr, &eptr);
      while (eptr != sptr) {
        ++j;
        sptr = eptr;
        parse_double(sptr, &eptr);
      }
      cnt[l] = j;
    }
  });
  // the column-count rule of src/io.c:171-199, in line order
  size_t nrows = 0, ncols = 0;
  std::vector<size_t> off(nl, 0);
  size_t k = 0;
  for (size_t l = 0; l < nl; ++l) {
    if (cnt[l] == kComment) continue;
    const size_t j = cnt[l];
    if (ncols == 0) {
      ncols = j;
    } else if (j == 0) {
      set_error("invalid line in grid matrix file: %zu", nrows + 1);
      return GOOSEBERRY_ERROR_INVALIDINPUT;
    } else if (j != ncols) {
      set_error("different number of columns (%zu) for line %zu when previous had %zu columns",
          j, nrows, ncols);
      return GOOSEBERRY_ERROR_INVALIDINPUT;
    }
    off[l] = k;
    k += j;
    ++nrows;
  }
  GB_CHECK_INPUT(nrows < 0xffffffffu && ncols < 0xffffffffu, "grid too large for 32-bit sizes");
  T * rowval = static_cast<T *>(std::calloc(nrows * ncols ? nrows * ncols : 1, sizeof(T)));
  if (!rowval) {
    set_error("out of host memory reading '%s'", path);
    return GOOSEBERRY_ERROR_UNKNOWN;
  }
  parallel_for(nt, [&](unsigned t) {
    for (size_t l = nl * t / nt; l < nl * (t + 1) / nt; ++l) {
      if (cnt[l] == kComment || cnt[l] == 0) continue;
      const char * sptr = L.buf.get() + L.start[l];
      char * eptr = nullptr;
      size_t q = off[l];
      double f = parse_double(sptr, &eptr);
      while (eptr != sptr) {
        rowval[q++] = static_cast<T>(f);
        sptr = eptr;
        f = parse_double(sptr, &eptr);
      }
    }
  });
  *r_rowval = rowval;
  *r_nrows = static_cast<dim_t>(nrows);
  *r_ncols = static_cast<dim_t>(ncols);
  return GOOSEBERRY_SUCCESS;
}

// printf's "%g" of v at o; returns the end.  std::to_chars with the general
// format and precision 6 is defined to give exactly printf's "%.6g"
// (C++17 [charconv.to.chars]) and is about twice as fast as snprintf;
// non-finite values keep snprintf's spelling ("inf", "-nan").
char * put_g(char * o, double v) {
  if (std::isfinite(v)) return std::to_chars(o, o + 32, v, std::chars_format::general, 6).ptr;
  char t[32];
  const int m = std::snprintf(t, sizeof t, "%g", v);
  std::memcpy(o, t, static_cast<size_t>(m));
  return o + m;
}

char * put_u(char * o, uint32_t v) { return std::to_chars(o, o + 16, v).ptr; }

// Most bytes one entry can take: a CSR pair (' ' + 10-digit column + ' ' +
// %g of at most 13 characters such as "-1.23457e-308"), or a grid value.
constexpr size_t kCsrEntryBytes = 26;
constexpr size_t kGridValueBytes = 16;

// Rows formatted by all threads and written in order.  The rows are cut into
// chunks of about 8 MiB (by each row's length bound); a thread takes the next
// chunk, formats it into its own buffer (reused from chunk to chunk) and
// writes it once the chunk before it is out.  Reused buffers stay warm:
// collecting each thread's whole share in one growing string first spent
// most of the time in first-touch page faults, which do not scale across
// threads.  row_bound(i) bounds the bytes of row i; fmt(i, o) writes row i at
// o and returns the end.
template <class Bound, class Fmt>
int write_rows(const char * path, size_t nrows, Bound && row_bound, Fmt && fmt) {
  GB_CHECK_INPUT(path != nullptr, "file name is NULL");
  FILE * f = std::fopen(path, "wb");
  if (!f) return open_error(path, "w");
  constexpr size_t kChunkBytes = size_t(8) << 20;
  std::vector<size_t> cut{0};  // chunk c holds rows [cut[c], cut[c + 1])
  std::vector<size_t> bound;   // bytes chunk c can take
  size_t acc = 0;
  for (size_t i = 0; i < nrows; ++i) {
    acc += row_bound(i);
    if (acc >= kChunkBytes || i + 1 == nrows) {
      cut.push_back(i + 1);
      bound.push_back(acc);
      acc = 0;
    }
  }
  const size_t nc = bound.size();
  const unsigned nt = static_cast<unsigned>(std::min<size_t>(n_threads(),
      std::max<size_t>(nc, 1)));
  std::atomic<size_t> next{0};
  std::mutex mu;
  std::condition_variable turn;
  size_t done = 0;          // chunks written (or passed over after an error); under mu
  bool io_ok = true, mem_ok = true;  // under mu
  parallel_for(nt, [&](unsigned) {
    std::unique_ptr<char[]> buf;
    size_t cap = 0;
    for (size_t c; (c = next.fetch_add(1)) < nc;) {
      if (bound[c] > cap) {
        buf.reset(new (std::nothrow) char[bound[c]]);
        cap = buf ? bound[c] : 0;
      }
      char * end = nullptr;
      if (buf) {
        end = buf.get();
        for (size_t i = cut[c]; i < cut[c + 1]; ++i) end = fmt(i, end);
      }
      // every chunk, failed or not, takes its turn so that later ones proceed
      std::unique_lock<std::mutex> lk(mu);
      turn.wait(lk, [&] { return done == c; });
      if (!end) {
        mem_ok = false;
      } else if (io_ok && mem_ok) {
        const size_t len = static_cast<size_t>(end - buf.get());
        io_ok = std::fwrite(buf.get(), 1, len, f) == len;
      }
      ++done;
      lk.unlock();
      turn.notify_all();
    }
  });
  io_ok = (std::fclose(f) == 0) && io_ok;
  if (!mem_ok) {
    set_error("out of host memory writing '%s'", path);
    return GOOSEBERRY_ERROR_UNKNOWN;
  }
  if (!io_ok) {
    set_error("write error on '%s'", path);
    return GOOSEBERRY_ERROR_WRITE;
  }
  return GOOSEBERRY_SUCCESS;
}

template <typename T>
int write_grid(const char * path, dim_t nrows, dim_t ncols, const T * rowval) {
  GB_CHECK_INPUT(nrows == 0 || ncols == 0 || rowval, "NULL values");
  return write_rows(path, nrows,
      [&](size_t) { return 1 + kGridValueBytes * static_cast<size_t>(ncols); },
      [&](size_t i, char * o) {
        for (dim_t j = 0; j < ncols; ++j) {
          if (j) *o++ = ' ';
          o = put_g(o, static_cast<double>(rowval[i * ncols + j]));
        }
        *o++ = '\n';
        return o;
      });
}

template <typename T>
int write_csr(const char * path, dim_t nrows, const ind_t * rowptr, const dim_t * rowind,
    const T * rowval) {
  GB_CHECK_INPUT(nrows == 0 || rowptr, "NULL rowptr");
  GB_CHECK_INPUT(nrows == 0 || rowptr[nrows] == 0 || (rowind && rowval), "NULL arrays");
  return write_rows(path, nrows,
      [&](size_t i) { return 1 + kCsrEntryBytes * static_cast<size_t>(rowptr[i + 1] - rowptr[i]); },
      [&](size_t i, char * o) {
        for (ind_t k = rowptr[i]; k < rowptr[i + 1]; ++k) {
          if (k != rowptr[i]) *o++ = ' ';
          o = put_u(o, static_cast<uint32_t>(rowind[k] + 1u));  // %u of the 1-based column
          *o++ = ' ';
          o = put_g(o, static_cast<double>(rowval[k]));
        }
        *o++ = '\n';
        return o;
      });
}

// The formats the reference reads and writes (src/io.c:1467-1545): CSR and
// GRID here; the others are recognised and reported as unimplemented.
int other_format(int type, bool sparse) {
  if (type == GOOSEBERRY_FORMAT_RAW || type == GOOSEBERRY_FORMAT_POINT ||
      type == GOOSEBERRY_FORMAT_SVM || type == GOOSEBERRY_FORMAT_GRAPH ||
      type == GOOSEBERRY_FORMAT_CLU || type == GOOSEBERRY_FORMAT_MATRIXMARKET ||
      type == (sparse ? GOOSEBERRY_FORMAT_GRID : GOOSEBERRY_FORMAT_CSR)) {
    set_error("%s matrix format %d is not implemented here (CSR and GRID are)",
        sparse ? "sparse" : "dense", type);
    return GOOSEBERRY_ERROR_UNIMPLEMENTED;
  }
  set_error("unrecognized %s matrix format '%d'", sparse ? "sparse" : "dense", type);
  return GOOSEBERRY_ERROR_INVALIDINPUT;
}

template <typename T>
int read_sparse(int type, const char * file, dim_t * nrows, dim_t * ncols, ind_t ** rowptr,
    dim_t ** rowind, T ** rowval) {
  if (type != GOOSEBERRY_FORMAT_CSR) return other_format(type, true);
  return read_csr<T>(file, nrows, ncols, rowptr, rowind, rowval,
      [](auto ** p, size_t n) {
        *p = malloc_n<std::remove_pointer_t<std::remove_pointer_t<decltype(p)>>>(n);
        return *p != nullptr;
      },
      [](void * p) { std::free(p); });
}

}  // namespace
}  // namespace gb

extern "C" {

int gooseberry_read_sparse_matrix(int type, const char * file, dim_t * nrows, dim_t * ncols,
    ind_t ** rowptr, dim_t ** rowind, float ** rowval) {
  return gb::read_sparse<float>(type, file, nrows, ncols, rowptr, rowind, rowval);
}

int gooseberry_read_sparse_matrix_f64(int type, const char * file, dim_t * nrows,
    dim_t * ncols, ind_t ** rowptr, dim_t ** rowind, double ** rowval) {
  return gb::read_sparse<double>(type, file, nrows, ncols, rowptr, rowind, rowval);
}

int gooseberry_read_dense_matrix(int type, const char * file, dim_t * nrows, dim_t * ncols,
    float ** rowval) {
  if (type != GOOSEBERRY_FORMAT_GRID) return gb::other_format(type, false);
  return gb::read_grid<float>(file, nrows, ncols, rowval);
}

int gooseberry_read_dense_matrix_f64(int type, const char * file, dim_t * nrows,
    dim_t * ncols, double ** rowval) {
  if (type != GOOSEBERRY_FORMAT_GRID) return gb::other_format(type, false);
  return gb::read_grid<double>(file, nrows, ncols, rowval);
}

int gooseberry_write_dense_matrix(int type, const char * file, dim_t nrows, dim_t ncols,
    const float * rowval) {
  if (type != GOOSEBERRY_FORMAT_GRID) return gb::other_format(type, false);
  return gb::write_grid<float>(file, nrows, ncols, rowval);
}

int gooseberry_write_dense_matrix_f64(int type, const char * file, dim_t nrows, dim_t ncols,
    const double * rowval) {
  if (type != GOOSEBERRY_FORMAT_GRID) return gb::other_format(type, false);
  return gb::write_grid<double>(file, nrows, ncols, rowval);
}

int gooseberry_write_sparse_matrix(int type, const char * file, dim_t nrows, dim_t ncols,
    const ind_t * rowptr, const dim_t * rowind, const float * rowval) {
  (void)ncols;
  if (type != GOOSEBERRY_FORMAT_CSR) return gb::other_format(type, true);
  return gb::write_csr<float>(file, nrows, rowptr, rowind, rowval);
}

int gooseberry_write_sparse_matrix_f64(int type, const char * file, dim_t nrows, dim_t ncols,
    const ind_t * rowptr, const dim_t * rowind, const double * rowval) {
  (void)ncols;
  if (type != GOOSEBERRY_FORMAT_CSR) return gb::other_format(type, true);
  return gb::write_csr<double>(file, nrows, rowptr, rowind, rowval);
}

// Parse a CSR file into host memory and upload it as a device matrix.
int gb_csr_read(const char * file, unsigned flags, gb_stream_t stream, gb_csr_t ** out) {
  GB_CHECK_INPUT(out != nullptr, "out is NULL");
  *out = nullptr;
  const bool want64 = (flags & GB_CSR_VALUES_F64) != 0;
  const bool want32 = (flags & GB_CSR_VALUES_F32) != 0;
  GB_CHECK_INPUT(want64 || want32, "flags must ask for GB_CSR_VALUES_F64 and/or _F32");
  GB_CHECK_INPUT((flags & GB_CSR_DEVICE_POINTERS) == 0,
      "gb_csr_read uploads its own copy; GB_CSR_DEVICE_POINTERS does not apply");
  std::vector<void *> held;
  auto alloc = [&](auto ** p, size_t n) {
    using E = std::remove_pointer_t<std::remove_pointer_t<decltype(p)>>;
    void * q = std::malloc(sizeof(E) * (n ? n : 1));
    if (!q) return false;
    held.push_back(q);
    *p = static_cast<E *>(q);
    return true;
  };
  dim_t nrows = 0, ncols = 0;
  ind_t * rowptr = nullptr;
  dim_t * rowind = nullptr;
  double * rowval = nullptr;
  auto release = [&](void * q) {
    held.erase(std::find(held.begin(), held.end(), q));
    std::free(q);
  };
  int rc = gb::read_csr<double>(file, &nrows, &ncols, &rowptr, &rowind, &rowval, alloc,
      release);
  if (rc == GOOSEBERRY_SUCCESS)
    rc = gb_csr_create(nrows, ncols, rowptr[nrows], rowptr, rowind, rowval, nullptr,
        (want64 ? GB_CSR_VALUES_F64 : 0u) | (want32 ? GB_CSR_VALUES_F32 : 0u), stream, out);
  if (rc == GOOSEBERRY_SUCCESS) cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  for (void * q : held) std::free(q);
  return rc;
}

}  // extern "C"
