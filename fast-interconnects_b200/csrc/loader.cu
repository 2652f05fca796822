// Relation files: the text format of the reference's file-backed join data
// (data-store/src/join_data.rs:173-260, JoinDataBuilder::build_with_files).
//
// A file holds one header line, then one tuple per line: the key and the
// payload as decimal integers separated by one space.  A file whose name
// ends in "gz" is gzip-compressed.  As in the reference, loading takes two
// passes over the file: one counts the tuples (so that the caller can size
// its columns), one parses them into the caller's key and payload columns.
//
// Host-only code (zlib for the compressed files); no GPU is touched.  Every
// malformed line is reported with its line number instead of being skipped:
// a record with other than two fields, a field that is not a decimal
// integer, or one outside the key type's range.  Empty lines (and a
// trailing carriage return) are ignored.
#include <zlib.h>

#include <cerrno>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../../include/fi_sqlops.h"
#include "api_internal.h"

namespace fi {
namespace {

bool ends_with_gz(const char *path) {
  const size_t n = std::strlen(path);
  return n >= 2 && path[n - 2] == 'g' && path[n - 1] == 'z';
}

// Line reader over a plain or gzip file (zlib reads both; a name ending in
// "gz" must hold gzip data, as the reference opens it with a gzip decoder).
class LineReader {
 public:
  ~LineReader() {
    if (f_) gzclose(f_);
  }
  int open(const char *path) {
    path_ = path;
    f_ = gzopen(path, "rb");
    if (!f_)
      return set_error(FI_ERR_INVALID_ARGUMENT, "cannot open %s: %s", path,
                       std::strerror(errno));
    gzbuffer(f_, 1u << 20);
    buf_.resize(1u << 20);
    if (fill() < 0) return FI_ERR_INVALID_ARGUMENT;
    if (ends_with_gz(path) && end_ > 0 && gzdirect(f_))
      return set_error(FI_ERR_INVALID_ARGUMENT, "%s: not gzip data", path);
    return FI_OK;
  }
  // Next line without its terminator; false at the end of the file, or on a
  // read error (then *rc is set).
  bool next(const char **b, const char **e, int *rc) {
    for (;;) {
      const char *start = buf_.data() + pos_;
      const char *stop = buf_.data() + end_;
      const char *nl = static_cast<const char *>(std::memchr(start, '\n', stop - start));
      if (nl) {
        pos_ = (size_t)(nl - buf_.data()) + 1;
        *b = start;
        *e = nl;
        ++line_;
        return true;
      }
      if (eof_) {
        if (start == stop) return false;
        pos_ = end_;  // last line without a newline
        *b = start;
        *e = stop;
        ++line_;
        return true;
      }
      // keep the partial line, refill behind it
      const size_t keep = end_ - pos_;
      if (keep == buf_.size()) buf_.resize(buf_.size() * 2);
      std::memmove(buf_.data(), start, keep);
      pos_ = 0;
      end_ = keep;
      if (fill() < 0) {
        *rc = FI_ERR_INVALID_ARGUMENT;
        return false;
      }
    }
  }
  uint64_t line() const { return line_; }

 private:
  int fill() {
    while (end_ < buf_.size() && !eof_) {
      const int n = gzread(f_, buf_.data() + end_, (unsigned)(buf_.size() - end_));
      if (n < 0) {
        int zerr = 0;
        const char *msg = gzerror(f_, &zerr);
        set_error(FI_ERR_INVALID_ARGUMENT, "%s: read error: %s", path_, msg);
        return -1;
      }
      if (n == 0) eof_ = true;
      end_ += (size_t)n;
    }
    return 0;
  }
  gzFile f_ = nullptr;
  const char *path_ = "";
  std::vector<char> buf_;
  size_t pos_ = 0, end_ = 0;
  bool eof_ = false;
  uint64_t line_ = 0;
};

// Trims a trailing carriage return; true for an empty line.
bool blank(const char *b, const char **e) {
  if (*e > b && (*e)[-1] == '\r') --*e;
  return *e == b;
}

// Decimal integer [b, e) with an optional sign into the range [lo, hi].
bool parse_int(const char *b, const char *e, int64_t lo, int64_t hi, int64_t *out) {
  if (b == e) return false;
  bool neg = false;
  if (*b == '-' || *b == '+') {
    neg = *b == '-';
    ++b;
    if (b == e) return false;
  }
  uint64_t v = 0;
  const uint64_t lim = neg ? (uint64_t)hi + 1 : (uint64_t)hi;  // |lo| = hi + 1
  for (; b < e; ++b) {
    const unsigned d = (unsigned)(*b - '0');
    if (d > 9) return false;
    if (v > (lim - d) / 10) return false;
    v = v * 10 + d;
  }
  *out = neg ? (int64_t)(0 - v) : (int64_t)v;
  return *out >= lo && *out <= hi;
}

template <typename K>
int read_file(const char *path, K *keys, K *pays, uint64_t len) {
  if (!path || (len && (!keys || !pays)))
    return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  LineReader r;
  int rc = r.open(path);
  if (rc) return rc;
  const char *b, *e;
  bool header = true;
  uint64_t n = 0;
  const int64_t lo = std::numeric_limits<K>::min(), hi = std::numeric_limits<K>::max();
  while (r.next(&b, &e, &rc)) {
    if (blank(b, &e)) continue;
    if (header) {  // the first line names the columns
      header = false;
      continue;
    }
    const char *sp = static_cast<const char *>(std::memchr(b, ' ', e - b));
    int64_t k, v;
    if (!sp || std::memchr(sp + 1, ' ', e - sp - 1))
      return set_error(FI_ERR_INVALID_ARGUMENT,
                       "%s:%llu: expected two fields separated by one space", path,
                       (unsigned long long)r.line());
    if (!parse_int(b, sp, lo, hi, &k) || !parse_int(sp + 1, e, lo, hi, &v))
      return set_error(FI_ERR_INVALID_ARGUMENT,
                       "%s:%llu: not a %d-bit integer key and payload", path,
                       (unsigned long long)r.line(), (int)(8 * sizeof(K)));
    if (keys) {
      if (n >= len)
        return set_error(FI_ERR_INVALID_ARGUMENT,
                         "%s holds more than %llu tuples", path,
                         (unsigned long long)len);
      keys[n] = (K)k;
      pays[n] = (K)v;
    }
    ++n;
  }
  if (rc) return rc;
  if (keys && n != len)
    return set_error(FI_ERR_INVALID_ARGUMENT, "%s holds %llu tuples, not %llu", path,
                     (unsigned long long)n, (unsigned long long)len);
  return FI_OK;
}

// Counting pass: lines after the header that are not empty.
int count_file(const char *path, uint64_t *len) {
  if (!path || !len) return set_error(FI_ERR_INVALID_ARGUMENT, "null argument");
  LineReader r;
  int rc = r.open(path);
  if (rc) return rc;
  const char *b, *e;
  bool header = true;
  uint64_t n = 0;
  while (r.next(&b, &e, &rc)) {
    if (blank(b, &e)) continue;
    if (header) {
      header = false;
      continue;
    }
    ++n;
  }
  if (rc) return rc;
  *len = n;
  return FI_OK;
}

}  // namespace
}  // namespace fi

extern "C" int fi_relation_file_len(const char *path, uint64_t *len) {
  return fi::count_file(path, len);
}

extern "C" int fi_relation_file_read_int32(const char *path, int32_t *keys,
                                           int32_t *pays, uint64_t len) {
  return fi::read_file<int32_t>(path, keys, pays, len);
}

extern "C" int fi_relation_file_read_int64(const char *path, int64_t *keys,
                                           int64_t *pays, uint64_t len) {
  return fi::read_file<int64_t>(path, keys, pays, len);
}
