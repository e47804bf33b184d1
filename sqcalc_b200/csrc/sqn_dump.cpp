// LAMMPS text dump ingest for the frame path: a multithreaded reader and a
// driver that parses the next frame while the GPU transforms the current one.
//
// The reader follows lammps_next_frame (src/sqc_dump.f90:162-313) and
// resolve_columns (:502-552): frames are "ITEM: TIMESTEP", "ITEM: NUMBER OF
// ATOMS", "ITEM: BOX BOUNDS [xy xz yz] ..." with three bound rows (two or three
// numbers each) and "ITEM: ATOMS <columns>" with one line per atom; the columns
// id, type and x|xu, y|yu, z|zu (case-insensitive, first match) are read in file
// order; a missing type or coordinate column is error 9.  Status of a failed
// read, as the reference's ierr: 4 malformed structure or TIMESTEP, 5 bad atom
// count, 6 bad BOX BOUNDS row, 7 ATOMS block before its header items, 8 short or
// malformed atom line, 9 missing column.
//
// B200-side design: the file is memory-mapped; one pass of memchr finds the end
// of the ATOMS block and the line where each thread starts, then the threads
// parse their lines with correctly rounded std::from_chars (the same doubles
// as any correctly rounding reader of the text).  The driver keeps two pinned
// host frames: while the plan uploads and transforms one, a host thread parses
// the next into the other.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cuda_runtime.h>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <charconv>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sqnufft.h"

struct sqn_dump_s {
  int fd = -1;
  const char *base = nullptr;
  size_t size = 0;
  size_t off = 0;
  int nthreads = 1;
  int last_error = 0;
  int64_t frames = 0;
  // pinned frames of sqn_accumulate_dump, kept for later calls (freed at close)
  double *pinned[2] = {nullptr, nullptr};
  int32_t *types = nullptr;
  int64_t pinned_atoms = 0;
};

namespace {

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// The line at off (without the newline); advances off past it.  False at EOF.
bool next_line(const sqn_dump *d, size_t &off, const char *&b, const char *&e) {
  if (off >= d->size) return false;
  b = d->base + off;
  const void *nl = std::memchr(b, '\n', d->size - off);
  e = nl ? static_cast<const char *>(nl) : d->base + d->size;
  off = (size_t)(e - d->base) + (nl ? 1 : 0);
  return true;
}

// Whitespace tokens of [b, e).
int tokens(const char *b, const char *e, std::vector<std::pair<const char *, const char *>> &out) {
  out.clear();
  const char *p = b;
  while (p < e) {
    while (p < e && is_space(*p)) ++p;
    if (p >= e) break;
    const char *s = p;
    while (p < e && !is_space(*p)) ++p;
    out.emplace_back(s, p);
  }
  return (int)out.size();
}

bool starts_item(const char *b, const char *e, const char *what) {
  const size_t n = std::strlen("ITEM: ");
  const size_t m = std::strlen(what);
  if ((size_t)(e - b) < n + m) return false;
  return std::memcmp(b, "ITEM: ", n) == 0 && std::memcmp(b + n, what, m) == 0;
}

bool parse_double(const char *b, const char *e, double &v) {
  if (b < e && *b == '+') ++b;
  auto r = std::from_chars(b, e, v);
  return r.ec == std::errc() && r.ptr == e;
}

// Exact powers of ten 1e0 .. 1e22 (every one is a double without rounding).
constexpr double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,
                               1e8,  1e9,  1e10, 1e11, 1e12, 1e13, 1e14, 1e15,
                               1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

// The leading decimal digits of the eight bytes at p (p + 8 <= the readable
// end): how many (0 .. 8) and their value.  With x = word ^ '0'...'0', a byte
// is a digit when x < 10: the lowest flagged byte of ((x + 0x76..) | x) &
// 0x80.. is the first non-digit (carries only flag bytes above it).  The
// digits are moved to the top of the word (leading zero digits below) and
// combined pairwise: 8 digits in three multiplications.
inline int digits8(const char *p, uint64_t &val) {
  uint64_t w;
  std::memcpy(&w, p, 8);
  const uint64_t x = w ^ 0x3030303030303030ull;
  const uint64_t m = ((x + 0x7676767676767676ull) | x) & 0x8080808080808080ull;
  const int n = m ? (__builtin_ctzll(m) >> 3) : 8;
  if (n == 0) {
    val = 0;
    return 0;
  }
  uint64_t y = n == 8 ? x : x << (8 * (8 - n));
  y = (y * 10) + (y >> 8);
  y = (((y & 0x000000FF000000FFull) * (100 + (1000000ull << 32))) +
       (((y >> 16) & 0x000000FF000000FFull) * (1 + (10000ull << 32)))) >> 32;
  val = y;
  return n;
}

constexpr uint64_t kPow10i[9] = {1, 10, 100, 1000, 10000, 100000, 1000000, 10000000,
                                 100000000};

// The same double as parse_double, faster for the plain decimals of a dump:
// when the digits form an integer w < 2^53 (at most 19 digits read) and the
// decimal exponent e satisfies |e| <= 22, w and 10^|e| are exact doubles and
// one IEEE multiplication or division rounds w * 10^e correctly (Clinger's
// fast path, W. D. Clinger, "How to read floating point numbers accurately",
// PLDI 1990).  Digits are read eight at a time while 8 bytes stay readable
// (before `lim`).  Anything else (more digits, larger exponents, inf, nan,
// stray characters) goes to std::from_chars.
bool parse_double_fast(const char *b, const char *e, const char *lim, double &v) {
  const char *p = b;
  bool neg = false;
  if (p < e && (*p == '+' || *p == '-')) neg = *p++ == '-';
  uint64_t w = 0;
  int nd = 0, e10 = 0;
  auto run = [&](bool frac) {
    for (;;) {
      int n;
      uint64_t val;
      if (p + 8 <= lim) {
        n = digits8(p, val);
        if (p + n > e) n = (int)(e - p), val = 0, nd = 99;  // digits past the token: give up
      } else {
        n = 0;
        val = 0;
        while (p + n < e && (unsigned)(p[n] - '0') < 10u && n < 8) val = val * 10 + (uint64_t)(p[n++] - '0');
      }
      if (n == 0) return;
      nd += n;
      if (nd <= 19) w = w * kPow10i[n] + val;
      if (frac) e10 -= n;
      p += n;
      if (n < 8) return;
    }
  };
  run(false);
  const bool int_digits = nd > 0;
  if (p < e && *p == '.') {
    ++p;
    run(true);
  }
  const bool digit = nd > 0 || int_digits;
  bool ok = nd <= 19;
  if (ok && digit && p < e && (*p == 'e' || *p == 'E')) {
    const char *q = p + 1;
    bool eneg = false;
    if (q < e && (*q == '+' || *q == '-')) eneg = *q++ == '-';
    int x = 0, nx = 0;
    for (; q < e && (unsigned)(*q - '0') < 10u && nx < 6; ++q, ++nx) x = x * 10 + (*q - '0');
    if (nx == 0) ok = false;
    e10 += eneg ? -x : x;
    p = q;
  }
  if (!(ok && digit && p == e && w < (1ull << 53) && e10 >= -22 && e10 <= 22))
    return parse_double(b, e, v);
  double r = (double)w;
  r = e10 >= 0 ? r * kPow10[e10] : r / kPow10[-e10];
  v = neg ? -r : r;
  return true;
}

bool parse_int(const char *b, const char *e, int64_t &v) {
  if (b < e && *b == '+') ++b;
  auto r = std::from_chars(b, e, v);
  if (r.ec == std::errc() && r.ptr == e) return true;
  double x;  // integers written as reals (e.g. "3.0")
  if (!parse_double(b, e, x) || x != (double)(int64_t)x) return false;
  v = (int64_t)x;
  return true;
}

// parse_int for the plain ids and types of a dump: up to eight digits read at
// once (8 bytes readable before lim), anything else through parse_int.
bool parse_int_fast(const char *b, const char *e, const char *lim, int64_t &v) {
  if (e - b <= 8 && e > b && b + 8 <= lim) {
    uint64_t val;
    if (b + digits8(b, val) == e) {
      v = (int64_t)val;
      return true;
    }
  }
  return parse_int(b, e, v);
}

std::string lower(const char *b, const char *e) {
  std::string s(b, e);
  for (char &c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

struct Columns {
  int id = -1, type = -1, x = -1, y = -1, z = -1, ncol = 0;
};

// The end of the token at q: the first ' ', '\t', '\r' or '\n' at or after q,
// or e.  Eight bytes at a time: the lowest flagged byte of
// (w - 0x21...) & ~w & 0x80... is the first byte below 0x21 (a borrow only
// flags bytes above a true one); other control bytes stay in the token.
const char *token_end(const char *q, const char *e) {
  for (;;) {
    while (q + 8 <= e) {
      uint64_t w;
      std::memcpy(&w, q, 8);
      const uint64_t m = (w - 0x2121212121212121ull) & ~w & 0x8080808080808080ull;
      if (m) {
        q += __builtin_ctzll(m) >> 3;
        break;
      }
      q += 8;
    }
    while (q < e && (unsigned char)*q > 0x20) ++q;
    if (q >= e || is_space(*q) || *q == '\n') return q;
    ++q;  // a control byte inside the token
  }
}

constexpr int kMaxActCols = 32;
inline int column_action(const Columns &c, int col, bool want_id) {
  if (col == c.x) return 1;
  if (col == c.y) return 2;
  if (col == c.z) return 3;
  if (col == c.type) return 4;
  if (want_id && col == c.id) return 5;
  return 0;
}

// Parse lines [first, first + count) of a block, the first starting at p: the
// columns are walked in one pass (a line needs at least ncol tokens; later
// tokens are ignored) and only id, type and the coordinates are converted.
int parse_lines(const char *p, const char *end, int64_t first, int64_t count, const Columns &c,
                double *pos, int32_t *type_id, int64_t *ids) {
  // what each column is: 1..3 a coordinate, 4 the type, 5 the id, 0 skipped
  int act_of[kMaxActCols];
  for (int k = 0; k < kMaxActCols; ++k) act_of[k] = column_action(c, k, ids != nullptr);
  for (int64_t i = first; i < first + count; ++i) {
    double xyz[3] = {0.0, 0.0, 0.0};
    int64_t t = 0, id = i + 1;
    const char *q = p;
    for (int col = 0; col < c.ncol; ++col) {
      while (q < end && is_space(*q)) ++q;
      if (q >= end || *q == '\n') return 8;
      const char *tb = q;
      q = token_end(q, end);
      const int act = col < kMaxActCols ? act_of[col] : column_action(c, col, ids != nullptr);
      if (act >= 1 && act <= 3) {
        if (!parse_double_fast(tb, q, end, xyz[act - 1])) return 8;
      } else if (act == 4) {
        if (!parse_int_fast(tb, q, end, t)) return 8;
      } else if (act == 5) {
        if (!parse_int_fast(tb, q, end, id)) return 8;
      }
    }
    pos[3 * i + 0] = xyz[0];
    pos[3 * i + 1] = xyz[1];
    pos[3 * i + 2] = xyz[2];
    type_id[i] = (int32_t)t;
    if (ids) ids[i] = id;
    const char *nl = static_cast<const char *>(std::memchr(q, '\n', (size_t)(end - q)));
    p = nl ? nl + 1 : end;
  }
  return 0;
}

// Newlines in [b, e): sixteen bytes at a time with SSE2 (x86-64's baseline),
// else eight at a time (for x = word ^ 0x0a0a..., a byte of x is zero exactly
// when the high bit of ((x & 0x7f..) + 0x7f..) | x is clear in it).
size_t count_newlines(const char *b, const char *e) {
  size_t n = 0;
  const char *p = b;
#if defined(__SSE2__)
  const __m128i nl = _mm_set1_epi8('\n');
  for (; p + 16 <= e; p += 16) {
    const __m128i v = _mm_loadu_si128(reinterpret_cast<const __m128i *>(p));
    n += (size_t)__builtin_popcount((unsigned)_mm_movemask_epi8(_mm_cmpeq_epi8(v, nl)));
  }
#else
  constexpr uint64_t kNl = 0x0a0a0a0a0a0a0a0aull, k7f = 0x7f7f7f7f7f7f7f7full;
  for (; p + 8 <= e; p += 8) {
    uint64_t w;
    std::memcpy(&w, p, 8);
    const uint64_t x = w ^ kNl;
    const uint64_t t = ((x & k7f) + k7f) | x;
    n += (size_t)__builtin_popcountll(~t & ~k7f);
  }
#endif
  for (; p < e; ++p) n += *p == '\n';
  return n;
}

// The position just past the n-th newline at or after `from` (n >= 1), or
// size when the file has fewer: whole 4 KB blocks are counted, the block
// holding the newline is scanned.
size_t nth_newline(const char *base, size_t size, size_t from, int64_t n) {
  size_t p = from;
  while (p < size) {
    const size_t q = std::min(size, p + 4096);
    const int64_t c = (int64_t)count_newlines(base + p, base + q);
    if (c < n) {
      n -= c;
      p = q;
      continue;
    }
    for (; p < q; ++p)
      if (base[p] == '\n' && --n == 0) return p + 1;
  }
  return size;
}

// One frame.  0 ok, 1 end of file (no further frame), 4-9 malformed.
int read_frame(sqn_dump *d, int64_t capacity, int64_t *natoms_out, int64_t *timestep,
               double *bounds, double *pos, int32_t *type_id, int64_t *ids) {
  size_t off = d->off;
  const char *b, *e;
  // skip to the next TIMESTEP item
  for (;;) {
    if (!next_line(d, off, b, e)) return 1;
    if (starts_item(b, e, "TIMESTEP")) break;
    // anything but blank lines before a frame is malformed
    const char *p = b;
    while (p < e && (is_space(*p))) ++p;
    if (p != e) return 4;
  }
  std::vector<std::pair<const char *, const char *>> tk;
  int64_t ts = 0, natoms = -1;
  bool have_box = false;
  double bx[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (!next_line(d, off, b, e) || tokens(b, e, tk) < 1 || !parse_int(tk[0].first, tk[0].second, ts))
    return 4;
  Columns c;
  for (;;) {
    if (!next_line(d, off, b, e)) return 4;
    if (starts_item(b, e, "NUMBER OF ATOMS")) {
      if (!next_line(d, off, b, e) || tokens(b, e, tk) < 1 ||
          !parse_int(tk[0].first, tk[0].second, natoms) || natoms <= 0)
        return 5;
    } else if (starts_item(b, e, "BOX BOUNDS")) {
      for (int k = 0; k < 3; ++k) {
        if (!next_line(d, off, b, e)) return 4;
        const int n = tokens(b, e, tk);
        if (n < 2) return 6;
        for (int m = 0; m < std::min(n, 3); ++m)
          if (!parse_double(tk[m].first, tk[m].second, bx[3 * k + m])) return 6;
      }
      have_box = true;
    } else if (starts_item(b, e, "ATOMS")) {
      if (natoms < 0 || !have_box) return 7;
      const int n = tokens(b, e, tk);
      c.ncol = n - 2;
      for (int m = 2; m < n; ++m) {
        const std::string name = lower(tk[m].first, tk[m].second);
        const int col = m - 2;
        if (name == "id" && c.id < 0) c.id = col;
        else if (name == "type" && c.type < 0) c.type = col;
        else if ((name == "x" || name == "xu") && c.x < 0) c.x = col;
        else if ((name == "y" || name == "yu") && c.y < 0) c.y = col;
        else if ((name == "z" || name == "zu") && c.z < 0) c.z = col;
      }
      if (c.type < 0 || c.x < 0 || c.y < 0 || c.z < 0) return 9;
      break;
    } else if (starts_item(b, e, "TIMESTEP")) {
      return 4;
    }
  }
  *natoms_out = natoms;
  if (natoms > capacity) return -1;  // caller's buffers too small
  // The ATOMS block: natoms lines from off.  Threads split a byte region that
  // should hold it (twice the first line's length per atom, widened when it
  // does not) and count the lines that start in their parts; a prefix over the
  // parts gives every part's first line index, the block end, and then the
  // threads parse the lines that start in their parts, all in parallel.
  int nt = (int)std::max<int64_t>(1, std::min<int64_t>(d->nthreads, natoms / 4096 + 1));
  const char *base = d->base;
  const size_t size = d->size;
  if (off >= size) return 8;
  // mean length of the first lines (up to 256), for the size of the region
  size_t len1;
  {
    size_t q = off;
    int64_t k = 0;
    for (; k < std::min<int64_t>(natoms, 256) && q < size; ++k) {
      const void *nl = std::memchr(base + q, '\n', size - q);
      q = nl ? (size_t)(static_cast<const char *>(nl) - base) + 1 : size;
    }
    len1 = std::max<size_t>(1, (q - off + (size_t)k - 1) / (size_t)std::max<int64_t>(k, 1));
  }
  auto run = [&](auto &&fn) {
    if (nt == 1) {
      fn(0);
      return;
    }
    std::vector<std::thread> th;
    for (int k = 1; k < nt; ++k) th.emplace_back(fn, k);
    fn(0);
    for (auto &t : th) t.join();
  };
  size_t region = std::min(size - off, (size_t)natoms * len1 / 8 * 9 + ((size_t)1 << 16));
  if (region < (size_t)nt * 4096) nt = 1;  // every part past the first starts 4 KB in
  std::vector<size_t> a((size_t)nt + 1);
  std::vector<int64_t> lines((size_t)nt), first((size_t)nt + 1);
  for (;;) {
    for (int k = 0; k <= nt; ++k) a[(size_t)k] = off + region * (size_t)k / (size_t)nt;
    // lines starting in [a_k, a_k+1): those after a newline in [a_k - 1, a_k+1 - 1)
    // (line 0 starts at off itself)
    run([&](int k) {
      const size_t lo = k == 0 ? off : a[(size_t)k] - 1, hi = a[(size_t)k + 1] - 1;
      lines[(size_t)k] = (k == 0 ? 1 : 0) + (int64_t)count_newlines(base + lo, base + std::max(lo, hi));
    });
    first[0] = 0;
    for (int k = 0; k < nt; ++k) first[(size_t)k + 1] = first[(size_t)k] + lines[(size_t)k];
    if (first[(size_t)nt] >= natoms || off + region == size) break;
    region = std::min(size - off, region * 2);
  }
  if (first[(size_t)nt] < natoms) return 8;  // the file ends inside the block
  // the block ends where line natoms starts: after the (natoms - first_j + 1)-th
  // newline from a_j - 1 for the part j holding line natoms - 1 (from off, the
  // natoms-th, for part 0), or at the end of the file
  size_t block_end;
  {
    int j = 0;
    while (first[(size_t)j + 1] <= natoms - 1) ++j;
    const size_t from = j == 0 ? off : a[(size_t)j] - 1;
    block_end = nth_newline(base, size, from, natoms - first[(size_t)j] + (j == 0 ? 0 : 1));
  }
  std::vector<int> err((size_t)nt, 0);
  run([&](int k) {
    const int64_t i0 = first[(size_t)k];
    const int64_t count = std::min<int64_t>(first[(size_t)k + 1], natoms) - i0;
    if (count <= 0) return;
    size_t q = off;
    if (k > 0) {
      const void *nl = std::memchr(base + a[(size_t)k] - 1, '\n', size - (a[(size_t)k] - 1));
      q = (size_t)(static_cast<const char *>(nl) - base) + 1;
    }
    err[(size_t)k] = parse_lines(base + q, base + block_end, i0, count, c, pos, type_id, ids);
  });
  for (int v : err)
    if (v) return v;
  *timestep = ts;
  if (bounds) std::memcpy(bounds, bx, sizeof(bx));
  d->off = block_end;
  d->frames++;
  return 0;
}

}  // namespace

extern "C" {

int sqn_dump_open(const char *path, int32_t nthreads, sqn_dump **out) {
  if (!out) return SQN_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!path) return SQN_ERR_INVALID_ARGUMENT;
  const int fd = ::open(path, O_RDONLY);
  if (fd < 0) return SQN_ERR_DUMP;
  struct stat sb;
  if (fstat(fd, &sb) != 0) {
    ::close(fd);
    return SQN_ERR_DUMP;
  }
  sqn_dump *d = new (std::nothrow) sqn_dump_s();
  if (!d) {
    ::close(fd);
    return SQN_ERR_ALLOC;
  }
  d->fd = fd;
  d->size = (size_t)sb.st_size;
  if (d->size > 0) {
    void *m = mmap(nullptr, d->size, PROT_READ, MAP_PRIVATE, fd, 0);
    if (m == MAP_FAILED) {
      ::close(fd);
      delete d;
      return SQN_ERR_DUMP;
    }
    madvise(m, d->size, MADV_SEQUENTIAL);
    d->base = static_cast<const char *>(m);
  }
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  d->nthreads = nthreads > 0 ? nthreads : (int)hw;
  *out = d;
  return SQN_OK;
}

int sqn_dump_next(sqn_dump *d, int64_t capacity, int64_t *natoms, int64_t *timestep,
                  double *bounds, double *pos, int32_t *type_id, int64_t *ids) {
  if (!d) return SQN_ERR_PLAN_NOTVALID;
  if (!natoms || !timestep || !pos || !type_id) return SQN_ERR_INVALID_ARGUMENT;
  *natoms = 0;
  *timestep = 0;
  const int r = read_frame(d, capacity, natoms, timestep, bounds, pos, type_id, ids);
  if (r == 1) {  // end of file: no frame, not an error
    *natoms = 0;
    d->last_error = 1;
    return SQN_OK;
  }
  if (r == -1) {
    d->last_error = 0;
    return SQN_ERR_INVALID_ARGUMENT;  // *natoms holds the count the buffers need
  }
  d->last_error = r;
  return r == 0 ? SQN_OK : SQN_ERR_DUMP;
}

int sqn_dump_last_error(const sqn_dump *d) { return d ? d->last_error : 3; }

int sqn_dump_rewind(sqn_dump *d) {
  if (!d) return SQN_ERR_PLAN_NOTVALID;
  d->off = 0;
  d->frames = 0;
  d->last_error = 0;
  return SQN_OK;
}

int sqn_dump_close(sqn_dump *d) {
  if (!d) return SQN_ERR_PLAN_NOTVALID;
  for (double *b : d->pinned)
    if (b) cudaFreeHost(b);
  std::free(d->types);
  if (d->base) munmap(const_cast<char *>(d->base), d->size);
  if (d->fd >= 0) ::close(d->fd);
  delete d;
  return SQN_OK;
}

int sqn_accumulate_dump(sqn_plan *plan, sqn_dump *d, int64_t max_frames,
                        const double *ref_bounds, int64_t *frames_done) {
  if (!plan || !d) return SQN_ERR_PLAN_NOTVALID;
  if (frames_done) *frames_done = 0;
  double ref[9];
  bool have_ref = ref_bounds != nullptr;
  if (have_ref) std::memcpy(ref, ref_bounds, sizeof(ref));
  sqn_plan_info info;
  int st = sqn_plan_info_get(plan, &info);
  if (st) return st;
  const int64_t cap = info.natoms;  // every frame must hold the plan's atoms
  if (cap <= 0) return SQN_ERR_PLAN_NOTVALID;
  if (d->pinned_atoms < cap) {
    for (double *&b : d->pinned)
      if (b) {
        cudaFreeHost(b);
        b = nullptr;
      }
    std::free(d->types);
    d->types = nullptr;
    d->pinned_atoms = 0;
    if (cudaMallocHost(&d->pinned[0], sizeof(double) * 3 * (size_t)cap) != cudaSuccess ||
        cudaMallocHost(&d->pinned[1], sizeof(double) * 3 * (size_t)cap) != cudaSuccess) {
      cudaGetLastError();
      return SQN_ERR_ALLOC;
    }
    d->types = static_cast<int32_t *>(std::malloc(sizeof(int32_t) * (size_t)cap));
    if (!d->types) return SQN_ERR_ALLOC;
    d->pinned_atoms = cap;
  }
  double *buf[2] = {d->pinned[0], d->pinned[1]};
  int32_t *types = d->types;
  // Parser thread: fills buffer k, then waits until the main thread has handed
  // that buffer to the plan (sqn_accumulate_frames returns once it has been read).
  std::mutex mu;
  std::condition_variable cv;
  int ready[2] = {0, 0};      // 1: parsed frame waiting, 2: end of input, <0: error
  bool free_[2] = {true, true};
  bool stop = false;
  int64_t limit = max_frames < 0 ? INT64_MAX : max_frames;
  std::thread parser([&]() {
    int k = 0;
    for (int64_t f = 0;; ++f) {
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return free_[k] || stop; });
        if (stop) return;
        free_[k] = false;
      }
      int code = 1;
      if (f < limit) {
        int64_t n = 0, ts = 0;
        double bx[9];
        const int r = sqn_dump_next(d, cap, &n, &ts, bx, buf[k], types, nullptr);
        if (r == SQN_ERR_INVALID_ARGUMENT && n > cap) {
          code = -SQN_ERR_NUM_NU_PTS_INVALID;  // more atoms than the plan
        } else if (r != SQN_OK) {
          code = -r;
        } else if (n == 0) {
          code = 2;
        } else if (n != cap) {
          code = -SQN_ERR_NUM_NU_PTS_INVALID;
        } else {
          // the box must not change between frames (relative 1e-6)
          if (!have_ref) {
            std::memcpy(ref, bx, sizeof(ref));
            have_ref = true;
          }
          double scale = 1.0, dev = 0.0;
          for (int i = 0; i < 9; ++i) {
            scale = std::max(scale, std::fabs(ref[i]));
            dev = std::max(dev, std::fabs(bx[i] - ref[i]));
          }
          if (dev > 1e-6 * scale) {
            d->last_error = 10;
            code = -SQN_ERR_DUMP;
          }
        }
      } else {
        code = 2;
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        ready[k] = code;
      }
      cv.notify_all();
      if (code != 1) return;
      k ^= 1;
    }
  });
  int k = 0;
  int64_t done = 0;
  for (;;) {
    int code;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv.wait(lk, [&] { return ready[k] != 0; });
      code = ready[k];
      ready[k] = 0;
    }
    if (code != 1) {
      if (code < 0) st = -code;
      break;
    }
    st = sqn_accumulate_frames(plan, buf[k], 1, SQN_HOST);
    {
      std::lock_guard<std::mutex> lk(mu);
      free_[k] = true;
      if (st != SQN_OK) stop = true;
    }
    cv.notify_all();
    if (st != SQN_OK) break;
    ++done;
    k ^= 1;
  }
  {
    std::lock_guard<std::mutex> lk(mu);
    stop = true;
  }
  cv.notify_all();
  parser.join();
  if (frames_done) *frames_done = done;
  const int sync = sqn_sync(plan);
  return st != SQN_OK ? st : sync;
}

}  // extern "C"
