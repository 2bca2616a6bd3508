// Oracle (test infrastructure only): text input helpers that restate the
// Fortran I/O semantics the reference relies on.
//
//  * PARSE (PARSE.f90:6-161, moduleparsing.f90): an 80-column line is split on
//    blanks/tabs; text between '#' and the next '#' (or end of line) is a
//    comment; column 80 is forced blank.
//  * list-directed READ(u,*): every READ starts at a new record, takes as many
//    values as it needs (continuing onto following records) and discards the
//    rest of the last record it touched.  Values are separated by blanks, tabs
//    or commas; 'D' exponents are accepted.  REAL*4 items are converted with
//    correct rounding (strtof), INTEGER items with strtol.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <fstream>
#include <sstream>

namespace orc {

inline std::string fix_exponent(std::string s) {
  for (auto& c : s) if (c == 'D' || c == 'd') c = 'E';
  return s;
}

inline bool parse_float(const std::string& tok, float* out) {
  std::string s = fix_exponent(tok);
  char* end = nullptr;
  errno = 0;
  float v = std::strtof(s.c_str(), &end);
  if (end == s.c_str() || *end != '\0') return false;
  *out = v;
  return true;
}
inline bool parse_double(const std::string& tok, double* out) {
  std::string s = fix_exponent(tok);
  char* end = nullptr;
  double v = std::strtod(s.c_str(), &end);
  if (end == s.c_str() || *end != '\0') return false;
  *out = v;
  return true;
}
inline bool parse_int(const std::string& tok, int* out) {
  char* end = nullptr;
  long v = std::strtol(tok.c_str(), &end, 10);
  if (end == tok.c_str() || *end != '\0') return false;
  *out = (int)v;
  return true;
}

// PARSE.f90: returns the words of an 80-column record.
inline std::vector<std::string> parse_line(const std::string& raw) {
  std::string line = raw.substr(0, std::min<size_t>(raw.size(), 80));
  if (line.size() == 80) line[79] = ' ';
  std::vector<std::string> words;
  size_t i = 0, n = line.size();
  while (i < n) {
    char c = line[i];
    if (c == '#') {
      size_t j = line.find('#', i + 1);
      if (j == std::string::npos) break;
      i = j + 1;
      continue;
    }
    if (c == ' ' || c == '\t' || c == '\r') { ++i; continue; }
    size_t b = i;
    while (i < n && line[i] != ' ' && line[i] != '\t' && line[i] != '\r' && line[i] != '#') ++i;
    words.push_back(line.substr(b, i - b));
    if (i < n && line[i] == '#') {
      size_t j = line.find('#', i + 1);
      if (j == std::string::npos) break;
      i = j + 1;
    }
  }
  return words;
}

// Tokens of a record for list-directed input (blank, tab and comma separate).
inline std::vector<std::string> ld_tokens(const std::string& line) {
  std::vector<std::string> t;
  size_t i = 0, n = line.size();
  while (i < n) {
    char c = line[i];
    if (c == ' ' || c == '\t' || c == ',' || c == '\r' || c == '\n') { ++i; continue; }
    if (c == '/') break;  // list-directed terminator
    size_t b = i;
    while (i < n && line[i] != ' ' && line[i] != '\t' && line[i] != ',' && line[i] != '\r' && line[i] != '\n') ++i;
    t.push_back(line.substr(b, i - b));
  }
  return t;
}

// A sequential formatted unit.
class Unit {
 public:
  bool open(const std::string& path) {
    std::ifstream f(path);
    if (!f) return false;
    std::string l;
    lines_.clear();
    while (std::getline(f, l)) lines_.push_back(l);
    pos_ = 0;
    return true;
  }
  bool eof() const { return pos_ >= lines_.size(); }
  void rewind() { pos_ = 0; }
  // READ(u,'(A80)') LINE
  bool read_a80(std::string* out) {
    if (pos_ >= lines_.size()) return false;
    *out = lines_[pos_++];
    return true;
  }
  // READ(u,*) with no items: skip one record.
  bool skip() {
    if (pos_ >= lines_.size()) return false;
    ++pos_;
    return true;
  }
  // READ(u,*) of n items: returns false at end of file before n items were read.
  bool read_items(size_t n, std::vector<std::string>* out) {
    out->clear();
    if (pos_ >= lines_.size()) return false;
    while (out->size() < n) {
      if (pos_ >= lines_.size()) return false;
      auto t = ld_tokens(lines_[pos_++]);
      for (auto& s : t) {
        if (out->size() < n) out->push_back(s);
      }
    }
    return true;
  }
  size_t nlines() const { return lines_.size(); }

 private:
  std::vector<std::string> lines_;
  size_t pos_ = 0;
};

}  // namespace orc
