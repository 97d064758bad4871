// textio.h -- the reference's text formats, shared by the drop-in executables.
//
//   B.txt        first token npix, then npix floats      (vissgen3d_blockage.cu:225-234)
//   theta/phi    npix floats, no header                  (:229-234)
//   uvw/xyza/xyzb  first row (3 tokens) skipped, then rows "a b c"   (:312-373)
//   bll          first token skipped, then one float per row         (:376-390)
//   C{d}day1M.txt  one float per line, default ostream precision     (:542-553)
// A missing input file reads as zero rows, as in the reference.
#pragma once

#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

namespace viss_host {

// Fast whitespace-separated float reader (the reference's ifstream >> float).
class TokenReader {
 public:
  explicit TokenReader(const std::string &path) {
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return;
    ok_ = true;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf_.resize(n > 0 ? static_cast<size_t>(n) + 1 : 1, '\0');
    if (n > 0 && std::fread(&buf_[0], 1, static_cast<size_t>(n), f) != static_cast<size_t>(n)) ok_ = false;
    std::fclose(f);
    p_ = buf_.c_str();
  }
  bool is_open() const { return ok_; }
  // next token as float; false at end of data or on a malformed token
  bool next(float &v) {
    if (!ok_) return false;
    while (*p_ == ' ' || *p_ == '\n' || *p_ == '\r' || *p_ == '\t') ++p_;
    if (!*p_) return false;
    char *end = nullptr;
    v = std::strtof(p_, &end);
    if (end == p_) return false;
    p_ = end;
    return true;
  }
  bool next_int(int &v) {
    float f;
    if (!next(f)) return false;
    v = static_cast<int>(f);
    return true;
  }

 private:
  std::string buf_;
  const char *p_ = nullptr;
  bool ok_ = false;
};

// "a b c" rows after a skipped first row; returns the row count.
inline long read_rows3(const std::string &path, std::vector<float> &a, std::vector<float> &b,
                       std::vector<float> &c) {
  TokenReader r(path);
  a.clear(); b.clear(); c.clear();
  if (!r.is_open()) return 0;
  float x, y, z;
  if (!(r.next(x) && r.next(y) && r.next(z))) return 0;  // first row, skipped
  while (r.next(x) && r.next(y) && r.next(z)) {
    a.push_back(x); b.push_back(y); c.push_back(z);
  }
  return static_cast<long>(a.size());
}

// one float per row after a skipped first token
inline long read_rows1(const std::string &path, std::vector<float> &a) {
  TokenReader r(path);
  a.clear();
  if (!r.is_open()) return 0;
  float x;
  if (!r.next(x)) return 0;
  while (r.next(x)) a.push_back(x);
  return static_cast<long>(a.size());
}

// one float per line, default ostream formatting (6 significant digits)
inline bool write_column(const std::string &path, const std::vector<float> &v) {
  std::ofstream f(path);
  if (!f.is_open()) return false;
  for (float x : v) f << x << '\n';
  return static_cast<bool>(f);
}

}  // namespace viss_host
