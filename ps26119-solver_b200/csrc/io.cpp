// io.cpp — see io.hpp. The file formats follow the reference's readers and writer
// (src/io/lpm_reader.cpp, mps_reader.cpp, solution_writer.cpp) so that files round-trip between
// the two libraries; the code is this library's own.
#include "io.hpp"

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <sstream>
#include <string_view>
#include <unordered_map>

namespace b200 {

bool ModelInfo::has_integers() const {
  return std::any_of(is_integer.begin(), is_integer.end(), [](char c) { return c != 0; });
}

std::string fingerprint_hex(const Model& m) {
  char buf[17];
  std::snprintf(buf, sizeof buf, "%016llx", static_cast<unsigned long long>(m.fingerprint()));
  return buf;
}

namespace {

bool slurp(const std::string& path, std::string& text, std::string& error) {
  std::ifstream in(path, std::ios::binary);
  if (!in) {
    error = "cannot open " + path;
    return false;
  }
  std::ostringstream ss;
  ss << in.rdbuf();
  text = ss.str();
  return true;
}

std::string_view trim(std::string_view s) {
  while (!s.empty() && std::isspace(static_cast<unsigned char>(s.front()))) s.remove_prefix(1);
  while (!s.empty() && std::isspace(static_cast<unsigned char>(s.back()))) s.remove_suffix(1);
  return s;
}

std::vector<std::string_view> split_ws(std::string_view s) {
  std::vector<std::string_view> out;
  std::size_t i = 0;
  while (i < s.size()) {
    while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
    const std::size_t b = i;
    while (i < s.size() && !std::isspace(static_cast<unsigned char>(s[i]))) ++i;
    if (i > b) out.push_back(s.substr(b, i - b));
  }
  return out;
}

std::string upper(std::string_view s) {
  std::string u(s);
  for (char& c : u) c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
  return u;
}

// A number token: [+-]digits[.digits][(e|E|d|D)[+-]digits], ".5", "inf" / "infinity"; NaN is
// refused (a NaN coefficient must not make a model).
bool parse_number(std::string_view t, double& out) {
  std::string b(t);
  if (!b.empty() && b[0] == '+') b.erase(0, 1);
  if (b.empty()) return false;
  for (char& c : b)
    if (c == 'd' || c == 'D') c = 'e';
  std::string low = b;
  for (char& c : low) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
  const bool neg = low[0] == '-';
  const std::string body = neg ? low.substr(1) : low;
  if (body == "inf" || body == "infinity") {
    out = neg ? -kInf : kInf;
    return true;
  }
  if (body.empty() || !(std::isdigit(static_cast<unsigned char>(body[0])) || body[0] == '.')) return false;
  for (char c : body)
    if (!std::isdigit(static_cast<unsigned char>(c)) && c != '.' && c != 'e' && c != '+' && c != '-') return false;
  char* end = nullptr;
  errno = 0;
  out = std::strtod(b.c_str(), &end);
  return end == b.c_str() + b.size();
}

// ------------------------------------------------------------------------------- .lpm
class LineScanner {
 public:
  explicit LineScanner(const std::string& t) : s_(t) {}
  bool line(std::string_view& out) {
    if (pos_ >= s_.size()) return false;
    const std::size_t e = s_.find('\n', pos_);
    const std::size_t end = e == std::string::npos ? s_.size() : e;
    out = std::string_view(s_).substr(pos_, end - pos_);
    if (!out.empty() && out.back() == '\r') out.remove_suffix(1);
    pos_ = end + 1;
    ++line_;
    return true;
  }
  bool token(std::string_view& out) {
    while (pos_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[pos_]))) {
      if (s_[pos_] == '\n') ++line_;
      ++pos_;
    }
    if (pos_ >= s_.size()) return false;
    const std::size_t b = pos_;
    while (pos_ < s_.size() && !std::isspace(static_cast<unsigned char>(s_[pos_]))) ++pos_;
    out = std::string_view(s_).substr(b, pos_ - b);
    return true;
  }
  void end_line() {
    while (pos_ < s_.size() && s_[pos_] != '\n') ++pos_;
    if (pos_ < s_.size()) ++pos_, ++line_;
  }
  int line_no() const { return line_; }

 private:
  const std::string& s_;
  std::size_t pos_ = 0;
  int line_ = 0;
};

bool parse_lpm_double(std::string_view t, double& v) {
  std::string b(t);
  char* end = nullptr;
  v = std::strtod(b.c_str(), &end);
  return !b.empty() && end == b.c_str() + b.size() && !std::isnan(v);
}
bool parse_lpm_int(std::string_view t, long long& v) {
  std::string b(t);
  char* end = nullptr;
  v = std::strtoll(b.c_str(), &end, 10);
  return !b.empty() && end == b.c_str() + b.size();
}

}  // namespace

bool read_lpm_text(const std::string& text, Model& M, ModelInfo& info, std::string& error) {
  M = Model{};
  info = ModelInfo{};
  LineScanner sc(text);
  auto fail = [&](const std::string& why) {
    error = "line " + std::to_string(sc.line_no()) + ": " + why;
    return false;
  };
  std::string_view ln;
  if (!sc.line(ln) || trim(ln) != "LPM 1") return fail("expected header 'LPM 1'");
  long long rows = -1, cols = -1, nnz = -1;
  constexpr long long kReserveCap = 1LL << 22;  // a bogus count must not allocate gigabytes
  auto doubles = [&](std::vector<double>& out, long long count) {
    out.clear();
    out.reserve(static_cast<std::size_t>(std::min(count, kReserveCap)));
    std::string_view t;
    double x;
    for (long long k = 0; k < count; ++k) {
      if (!sc.token(t) || !parse_lpm_double(t, x)) return false;
      out.push_back(x);
    }
    sc.end_line();
    return true;
  };
  auto ints = [&](std::vector<int>& out, long long count) {
    out.clear();
    out.reserve(static_cast<std::size_t>(std::min(count, kReserveCap)));
    std::string_view t;
    long long v;
    for (long long k = 0; k < count; ++k) {
      if (!sc.token(t) || !parse_lpm_int(t, v) || v < std::numeric_limits<int>::min() ||
          v > std::numeric_limits<int>::max())
        return false;
      out.push_back(static_cast<int>(v));
    }
    sc.end_line();
    return true;
  };
  bool ended = false;
  while (sc.line(ln)) {
    const std::string_view t = trim(ln);
    if (t.empty() || t.front() == '#') continue;
    const std::size_t sp = t.find(' ');
    const std::string_view tag = t.substr(0, sp);
    const std::string_view rest = sp == std::string_view::npos ? std::string_view{} : trim(t.substr(sp + 1));
    const bool sized = rows >= 0 && cols >= 0 && nnz >= 0;
    if (tag == "END") {
      ended = true;
      break;
    } else if (tag == "NAME") {
      info.name = std::string(rest);
    } else if (tag == "SENSE") {
      if (rest == "MIN") M.sense = 1;
      else if (rest == "MAX") M.sense = -1;
      else return fail("SENSE must be MIN or MAX");
    } else if (tag == "ROWS" || tag == "COLS" || tag == "NNZ") {
      long long v;
      if (!parse_lpm_int(rest, v) || v < 0 || v > std::numeric_limits<int>::max()) return fail("bad size");
      (tag == "ROWS" ? rows : tag == "COLS" ? cols : nnz) = v;
    } else if (tag == "OFFSET") {
      if (!parse_lpm_double(rest, M.obj_offset)) return fail("bad OFFSET");
    } else if (!sized) {
      return fail("ROWS/COLS/NNZ must precede section " + std::string(tag));
    } else if (tag == "OBJ") {
      if (!doubles(M.obj, cols)) return fail("bad OBJ section");
    } else if (tag == "COL_LOWER") {
      if (!doubles(M.col_lower, cols)) return fail("bad COL_LOWER section");
    } else if (tag == "COL_UPPER") {
      if (!doubles(M.col_upper, cols)) return fail("bad COL_UPPER section");
    } else if (tag == "ROW_LOWER") {
      if (!doubles(M.row_lower, rows)) return fail("bad ROW_LOWER section");
    } else if (tag == "ROW_UPPER") {
      if (!doubles(M.row_upper, rows)) return fail("bad ROW_UPPER section");
    } else if (tag == "COL_START") {
      if (!ints(M.col_start, cols + 1)) return fail("bad COL_START section");
    } else if (tag == "ROW_INDEX") {
      if (!ints(M.row_index, nnz)) return fail("bad ROW_INDEX section");
    } else if (tag == "VALUE") {
      if (!doubles(M.value, nnz)) return fail("bad VALUE section");
    } else if (tag == "INTEGER") {
      std::vector<int> v;
      if (!ints(v, cols)) return fail("bad INTEGER section");
      info.is_integer.assign(v.begin(), v.end());
    } else if (tag == "ROW_NAMES" || tag == "COL_NAMES") {
      auto& names = tag == "ROW_NAMES" ? info.row_names : info.col_names;
      const long long count = tag == "ROW_NAMES" ? rows : cols;
      for (long long k = 0; k < count; ++k) {
        if (!sc.line(ln)) return fail("unexpected end of names");
        names.emplace_back(ln);
      }
    } else {
      return fail("unknown section '" + std::string(tag) + "'");
    }
  }
  if (!ended) return fail("missing END");
  if (rows < 0 || cols < 0 || nnz < 0) return fail("missing ROWS/COLS/NNZ");
  M.num_rows = static_cast<int>(rows);
  M.num_cols = static_cast<int>(cols);
  if (M.col_start.empty() && cols == 0) M.col_start = {0};
  M.is_integer = info.is_integer;
  if (auto err = M.validate(); !err.empty()) return fail("invalid model: " + err);
  return true;
}

bool read_lpm(const std::string& path, Model& M, ModelInfo& info, std::string& error) {
  std::string text;
  return slurp(path, text, error) && read_lpm_text(text, M, info, error);
}

bool write_lpm(const std::string& path, const Model& m, const ModelInfo& info, std::string& error) {
  std::FILE* f = std::fopen(path.c_str(), "w");
  if (!f) {
    error = "cannot open " + path + " for writing";
    return false;
  }
  auto num = [&](double v) {
    if (v == kInf) std::fputs("inf", f);
    else if (v == -kInf) std::fputs("-inf", f);
    else std::fprintf(f, "%.17g", v);
  };
  auto dvec = [&](const char* tag, const std::vector<double>& v) {
    std::fprintf(f, "%s\n", tag);
    for (std::size_t k = 0; k < v.size(); ++k) {
      num(v[k]);
      std::fputc((k % 8 == 7 || k + 1 == v.size()) ? '\n' : ' ', f);
    }
  };
  auto ivec = [&](const char* tag, const auto& v) {
    std::fprintf(f, "%s\n", tag);
    for (std::size_t k = 0; k < v.size(); ++k)
      std::fprintf(f, "%d%c", static_cast<int>(v[k]), (k % 16 == 15 || k + 1 == v.size()) ? '\n' : ' ');
  };
  std::fprintf(f, "LPM 1\n# fingerprint %s\nNAME %s\nSENSE %s\nROWS %d\nCOLS %d\nNNZ %zu\nOFFSET ",
               fingerprint_hex(m).c_str(), info.name.c_str(), m.sense == -1 ? "MAX" : "MIN", m.num_rows, m.num_cols,
               m.nnz());
  num(m.obj_offset);
  std::fputc('\n', f);
  dvec("OBJ", m.obj);
  dvec("COL_LOWER", m.col_lower);
  dvec("COL_UPPER", m.col_upper);
  dvec("ROW_LOWER", m.row_lower);
  dvec("ROW_UPPER", m.row_upper);
  ivec("COL_START", m.col_start);
  ivec("ROW_INDEX", m.row_index);
  dvec("VALUE", m.value);
  if (!info.is_integer.empty()) ivec("INTEGER", info.is_integer);
  if (!info.row_names.empty()) {
    std::fputs("ROW_NAMES\n", f);
    for (const auto& s : info.row_names) std::fprintf(f, "%s\n", s.c_str());
  }
  if (!info.col_names.empty()) {
    std::fputs("COL_NAMES\n", f);
    for (const auto& s : info.col_names) std::fprintf(f, "%s\n", s.c_str());
  }
  std::fputs("END\n", f);
  const bool ok = std::fclose(f) == 0;
  if (!ok) error = "write failed for " + path;
  return ok;
}

// -------------------------------------------------------------------------------- MPS
namespace {

struct MpsError {
  std::string what;
};

class MpsParser {
 public:
  explicit MpsParser(bool fixed) : fixed_(fixed) {}

  void parse(std::string_view text) {
    std::size_t pos = 0;
    while (pos < text.size() && section_ != kEndata) {
      std::size_t e = text.find('\n', pos);
      if (e == std::string_view::npos) e = text.size();
      std::string_view ln = text.substr(pos, e - pos);
      pos = e + 1;
      ++line_;
      if (!ln.empty() && ln.back() == '\r') ln.remove_suffix(1);
      line(ln);
    }
  }
  void finish(Model& M, ModelInfo& info);

 private:
  enum Section { kNone, kName, kObjSense, kObjName, kRows, kColumns, kRhs, kRanges, kBounds, kEndata };
  enum RowType { kE, kL, kG };
  static constexpr int kObjective = -1, kFreeRow = -2;

  [[noreturn]] void fail(const std::string& why) const { throw MpsError{"line " + std::to_string(line_) + ": " + why}; }
  void warn(const std::string& why) { warnings_.push_back("line " + std::to_string(line_) + ": " + why); }
  double number(std::string_view t) const {
    double v;
    if (!parse_number(t, v)) fail("expected a number, found '" + std::string(t) + "'");
    return v;
  }
  static double as_inf(double v) { return v >= 1e30 ? kInf : (v <= -1e30 ? -kInf : v); }
  static std::string_view field(std::string_view ln, int first, int last) {  // 1-based columns
    if (static_cast<int>(ln.size()) < first) return {};
    const std::size_t b = static_cast<std::size_t>(first - 1);
    return trim(ln.substr(b, std::min<std::size_t>(static_cast<std::size_t>(last - first + 1), ln.size() - b)));
  }
  int row_of(std::string_view name) const {
    const auto it = rows_.find(std::string(name));
    if (it == rows_.end()) fail("unknown row '" + std::string(name) + "'");
    return it->second;
  }
  int col_of(std::string_view name) const {
    const auto it = cols_.find(std::string(name));
    if (it == cols_.end()) fail("unknown column '" + std::string(name) + "'");
    return it->second;
  }
  // several RHS / RANGES / BOUNDS vectors may be given; the first one named is used
  bool take_set(std::string& chosen, bool& have, std::string_view set, const char* what) {
    if (!have) {
      chosen = std::string(set), have = true;
      return true;
    }
    if (set == chosen) return true;
    if (!ignored_warned_) warn(std::string("ignoring additional ") + what + " set '" + std::string(set) + "'");
    ignored_warned_ = true;
    return false;
  }

  void line(std::string_view ln) {
    if (trim(ln).empty() || ln[0] == '*') return;
    const bool indented = ln[0] == ' ' || ln[0] == '\t';
    if (!indented && header(ln)) return;
    switch (section_) {
      case kObjSense: sense(split_ws(ln)[0]); break;
      case kObjName: objname_ = std::string(split_ws(ln)[0]); break;
      case kRows: row(ln); break;
      case kColumns: column(ln); break;
      case kRhs: rhs_range(ln, false); break;
      case kRanges: rhs_range(ln, true); break;
      case kBounds: bound(ln); break;
      default: fail("data line outside of any section");
    }
  }
  bool header(std::string_view ln) {
    const auto t = split_ws(ln);
    const std::string key = upper(t[0]);
    if (key == "NAME") {
      section_ = kName;
      name_ = std::string(trim(trim(ln).substr(4)));
    } else if (key == "OBJSENSE" || key == "OBJSENCE") {
      section_ = kObjSense;
      if (t.size() > 1) sense(t[1]);
    } else if (key == "OBJNAME") {
      section_ = kObjName;
      if (t.size() > 1) objname_ = std::string(t[1]);
    } else if (key == "ROWS") {
      section_ = kRows;
    } else if (key == "COLUMNS") {
      if (rows_.empty()) fail("COLUMNS section before any ROWS");
      section_ = kColumns;
    } else if (key == "RHS") {
      section_ = kRhs;
    } else if (key == "RANGES") {
      section_ = kRanges;
    } else if (key == "BOUNDS") {
      section_ = kBounds;
    } else if (key == "ENDATA") {
      section_ = kEndata;
      endata_ = true;
    } else if (key == "QUADOBJ" || key == "QMATRIX" || key == "QSECTION" || key == "QCMATRIX" || key == "SOS" ||
               key == "CSECTION" || key == "INDICATORS" || key == "CONES") {
      fail("section " + key + " is not supported (linear programs only)");
    } else if (!fixed_ && section_ >= kRows) {
      return false;  // an unindented data line, tolerated in free format
    } else {
      fail("unknown section '" + std::string(t[0]) + "'");
    }
    return true;
  }
  void sense(std::string_view tok) {
    const std::string s = upper(tok);
    if (s == "MAX" || s == "MAXIMIZE") sense_ = -1;
    else if (s == "MIN" || s == "MINIMIZE") sense_ = 1;
    else fail("unknown OBJSENSE '" + std::string(tok) + "'");
  }
  void row(std::string_view ln) {
    std::string_view type, name;
    if (!fixed_) {
      const auto t = split_ws(ln);
      if (t.size() != 2) fail("ROWS line needs exactly 2 fields (type, name)");
      type = t[0], name = t[1];
    } else {
      type = field(ln, 2, 3), name = field(ln, 5, 12);
    }
    if (name.empty()) fail("ROWS line without a row name");
    const std::string key(name);
    if (rows_.count(key)) fail("duplicate row name '" + key + "'");
    const std::string ty = upper(type);
    if (ty == "N") {  // the first N row (or the OBJNAME one) is the objective; others are dropped
      if (!have_obj_ && (objname_.empty() || objname_ == key)) {
        rows_[key] = kObjective;
        have_obj_ = true;
      } else {
        rows_[key] = kFreeRow;
        ++dropped_;
      }
      return;
    }
    RowType rt;
    if (ty == "E") rt = kE;
    else if (ty == "L") rt = kL;
    else if (ty == "G") rt = kG;
    else fail("unknown row type '" + std::string(type) + "'");
    rows_[key] = static_cast<int>(row_names_.size());
    row_names_.push_back(key);
    row_types_.push_back(rt);
    rhs_.push_back(0.0), range_.push_back(0.0), has_rhs_.push_back(0), has_range_.push_back(0);
  }
  void column(std::string_view ln) {
    if (ln.find('\'') != std::string_view::npos) {  // integer block markers: 'MARKER' 'INTORG' / 'INTEND'
      const std::string u = upper(ln);
      if (u.find("'MARKER'") != std::string::npos) {
        if (u.find("'INTORG'") != std::string::npos) in_int_ = true;
        else if (u.find("'INTEND'") != std::string::npos) in_int_ = false;
        else fail("MARKER line without 'INTORG' or 'INTEND'");
        return;
      }
    }
    const auto t = split_ws(ln);
    std::string_view col, r1, v1, r2, v2;
    if (!fixed_) {
      if (t.size() != 3 && t.size() != 5) fail("COLUMNS line needs 3 or 5 fields");
      col = t[0], r1 = t[1], v1 = t[2];
      if (t.size() == 5) r2 = t[3], v2 = t[4];
    } else {
      col = field(ln, 5, 12), r1 = field(ln, 15, 22), v1 = field(ln, 25, 36), r2 = field(ln, 40, 47),
      v2 = field(ln, 50, 61);
      if (col.empty() || r1.empty() || v1.empty()) fail("incomplete COLUMNS line");
    }
    const int j = column_index(col);
    coefficient(j, r1, number(v1));
    if (!r2.empty()) coefficient(j, r2, number(v2));
  }
  int column_index(std::string_view name) {
    if (current_ >= 0 && col_names_[current_] == name) return current_;
    const std::string key(name);
    const auto it = cols_.find(key);
    if (it != cols_.end()) {
      warn("entries of column '" + key + "' are not contiguous");
      return current_ = it->second;
    }
    current_ = static_cast<int>(col_names_.size());
    cols_[key] = current_;
    col_names_.push_back(key);
    obj_.push_back(0.0), lo_.push_back(0.0), up_.push_back(kInf);
    int_.push_back(in_int_ ? 1 : 0), lo_set_.push_back(0), up_set_.push_back(0);
    return current_;
  }
  void coefficient(int j, std::string_view row_name, double v) {
    const int i = row_of(row_name);
    if (!std::isfinite(v)) fail("coefficient of column '" + col_names_[j] + "' in row '" + std::string(row_name) +
                                "' is not finite");
    if (i == kObjective) obj_[j] += v;
    else if (i >= 0 && v != 0.0) trip_.push_back({j, i, v});
  }
  void rhs_range(std::string_view ln, bool range) {
    std::string_view set, r1, v1, r2, v2;
    if (!fixed_) {
      const auto t = split_ws(ln);
      std::size_t k = 0;
      if (t.size() == 3 || t.size() == 5) set = t[0], k = 1;
      else if (t.size() != 2 && t.size() != 4) fail(std::string(range ? "RANGES" : "RHS") + " line needs 2 to 5 fields");
      r1 = t[k], v1 = t[k + 1];
      if (t.size() - k == 4) r2 = t[k + 2], v2 = t[k + 3];
    } else {
      set = field(ln, 5, 12), r1 = field(ln, 15, 22), v1 = field(ln, 25, 36), r2 = field(ln, 40, 47),
      v2 = field(ln, 50, 61);
      if (r1.empty() || v1.empty()) fail("incomplete RHS/RANGES line");
    }
    const bool use = range ? take_set(range_set_, have_range_set_, set, "RANGES")
                           : take_set(rhs_set_, have_rhs_set_, set, "RHS");
    if (!use) return;
    rhs_entry(r1, number(v1), range);
    if (!r2.empty()) rhs_entry(r2, number(v2), range);
  }
  void rhs_entry(std::string_view row_name, double v, bool range) {
    const int i = row_of(row_name);
    if (i == kFreeRow) return;
    if (i == kObjective) {
      if (range) {
        warn("RANGES entry on the objective row ignored");
      } else {
        if (!std::isfinite(v)) fail("objective constant (RHS on the objective row) is not finite");
        offset_ = -v;  // an RHS on the objective is minus the objective constant
      }
      return;
    }
    if (range) {
      if (has_range_[i]) warn("row '" + row_names_[i] + "' has more than one RANGES entry; the last one is used");
      range_[i] = v, has_range_[i] = 1;
    } else {
      if (has_rhs_[i]) warn("row '" + row_names_[i] + "' has more than one RHS entry; the last one is used");
      rhs_[i] = v, has_rhs_[i] = 1;
    }
  }
  void bound(std::string_view ln) {
    std::string_view type, set, col, val;
    if (!fixed_) {
      const auto t = split_ws(ln);
      if (t.size() < 2) fail("BOUNDS line too short");
      type = t[0];
      const std::string ty = upper(type);
      const bool needs_value = ty == "UP" || ty == "LO" || ty == "FX" || ty == "LI" || ty == "UI";
      const std::size_t rest = t.size() - 1;
      if (needs_value) {
        if (rest == 3) set = t[1], col = t[2], val = t[3];
        else if (rest == 2) col = t[1], val = t[2];
        else fail("BOUNDS line of type " + ty + " needs a column and a value");
      } else {  // FR / MI / PL / BV: the value is optional; "BV X 1" vs "BV SET X" by column name
        double tmp;
        if (rest == 1) col = t[1];
        else if (rest == 2 && cols_.count(std::string(t[1])) && parse_number(t[2], tmp)) col = t[1], val = t[2];
        else if (rest == 2) set = t[1], col = t[2];
        else if (rest == 3) set = t[1], col = t[2], val = t[3];
        else fail("malformed BOUNDS line");
      }
    } else {
      type = field(ln, 2, 3), set = field(ln, 5, 12), col = field(ln, 15, 22), val = field(ln, 25, 36);
    }
    if (!take_set(bound_set_, have_bound_set_, set, "BOUNDS")) return;
    const int j = col_of(col);
    const std::string ty = upper(type);
    auto value = [&] { return as_inf(number(val)); };
    if (ty == "UP" || ty == "UI") {
      const double v = value();
      up_[j] = v, up_set_[j] = 1;
      if (v < 0.0 && lo_[j] == 0.0 && !lo_set_[j]) {  // negative upper bound with the default lower
        lo_[j] = -kInf;
        warn("negative upper bound on '" + col_names_[j] + "' with default lower bound: lower set to -inf");
      }
      if (ty == "UI") int_[j] = 1;
    } else if (ty == "LO" || ty == "LI") {
      lo_[j] = value(), lo_set_[j] = 1;
      if (ty == "LI") int_[j] = 1;
    } else if (ty == "FX") {
      const double v = value();
      lo_[j] = up_[j] = v, lo_set_[j] = up_set_[j] = 1;
    } else if (ty == "FR") {
      lo_[j] = -kInf, up_[j] = kInf, lo_set_[j] = up_set_[j] = 1;
    } else if (ty == "MI") {
      lo_[j] = -kInf, lo_set_[j] = 1;
    } else if (ty == "PL") {
      up_[j] = kInf, up_set_[j] = 1;
    } else if (ty == "BV") {
      lo_[j] = 0.0, up_[j] = 1.0, lo_set_[j] = up_set_[j] = 1, int_[j] = 1;
    } else if (ty == "SC") {
      fail("semi-continuous (SC) bounds are not supported");
    } else {
      fail("unknown bound type '" + std::string(type) + "'");
    }
  }

  struct Trip {
    int col, row;
    double v;
  };
  bool fixed_;
  int line_ = 0;
  Section section_ = kNone;
  bool endata_ = false, have_obj_ = false, in_int_ = false, ignored_warned_ = false;
  int dropped_ = 0, sense_ = 1, current_ = -1;
  double offset_ = 0.0;
  std::string name_, objname_;
  std::unordered_map<std::string, int> rows_, cols_;
  std::vector<std::string> row_names_, col_names_, warnings_;
  std::vector<RowType> row_types_;
  std::vector<double> rhs_, range_, obj_, lo_, up_;
  std::vector<char> has_rhs_, has_range_, int_, lo_set_, up_set_;
  std::vector<Trip> trip_;
  std::string rhs_set_, range_set_, bound_set_;
  bool have_rhs_set_ = false, have_range_set_ = false, have_bound_set_ = false;
};

void MpsParser::finish(Model& M, ModelInfo& info) {
  if (section_ == kNone) fail("no MPS section found (empty file or not an MPS file)");
  if (!endata_) warnings_.push_back("file ended without ENDATA");
  if (!have_obj_) warnings_.push_back("no objective (N) row found; objective is zero");
  if (dropped_ > 0) warnings_.push_back("dropped " + std::to_string(dropped_) + " extra free (N) row(s)");
  const int m = static_cast<int>(row_names_.size()), n = static_cast<int>(col_names_.size());
  // CSC with rows sorted inside each column; duplicate entries are summed, zero sums dropped
  std::stable_sort(trip_.begin(), trip_.end(),
                   [](const Trip& a, const Trip& b) { return a.col != b.col ? a.col < b.col : a.row < b.row; });
  M = Model{};
  M.num_rows = m, M.num_cols = n, M.sense = sense_, M.obj_offset = offset_;
  M.col_start.assign(static_cast<std::size_t>(n) + 1, 0);
  int merged = 0;
  std::size_t k = 0;
  for (int j = 0; j < n; ++j) {
    M.col_start[j] = static_cast<int>(M.value.size());
    while (k < trip_.size() && trip_[k].col == j) {
      const int r = trip_[k].row;
      double sum = trip_[k].v;
      for (++k; k < trip_.size() && trip_[k].col == j && trip_[k].row == r; ++k) sum += trip_[k].v, ++merged;
      if (sum != 0.0) M.row_index.push_back(r), M.value.push_back(sum);
    }
  }
  M.col_start[n] = static_cast<int>(M.value.size());
  if (merged > 0) warnings_.push_back("summed " + std::to_string(merged) + " duplicate matrix entries");
  M.obj = obj_;
  // row bounds from the type, RHS b and RANGES R:
  //   E: [b, b], R > 0: [b, b + |R|], R < 0: [b − |R|, b];   L: [−inf, b] or [b − |R|, b];
  //   G: [b, +inf] or [b, b + |R|]
  M.row_lower.resize(m), M.row_upper.resize(m);
  for (int i = 0; i < m; ++i) {
    const double b = as_inf(rhs_[i]), r = std::fabs(as_inf(range_[i]));
    double lo = 0.0, up = 0.0;
    switch (row_types_[i]) {
      case kE:
        lo = up = b;
        if (has_range_[i] && range_[i] > 0) up = b + r;
        if (has_range_[i] && range_[i] < 0) lo = b - r;
        break;
      case kL:
        lo = has_range_[i] ? b - r : -kInf;
        up = b;
        break;
      case kG:
        lo = b;
        up = has_range_[i] ? b + r : kInf;
        break;
    }
    M.row_lower[i] = lo, M.row_upper[i] = up;
  }
  for (int j = 0; j < n; ++j)
    if (lo_[j] > up_[j]) warnings_.push_back("column '" + col_names_[j] + "' has lower bound > upper bound");
  M.col_lower = lo_, M.col_upper = up_;
  info = ModelInfo{};
  info.name = name_;
  info.row_names = row_names_;
  info.col_names = col_names_;
  info.is_integer = int_;
  info.warnings = warnings_;
  M.is_integer = int_;
}

}  // namespace

bool read_mps_text(const std::string& text, Model& M, ModelInfo& info, std::string& error) {
  // free format reads almost every file; fixed format is needed only when names contain spaces
  try {
    MpsParser p(false);
    p.parse(text);
    p.finish(M, info);
  } catch (const MpsError& free_err) {
    try {
      MpsParser p(true);
      p.parse(text);
      p.finish(M, info);
      info.warnings.insert(info.warnings.begin(),
                           "free-format parse failed (" + free_err.what + "); file was read as fixed format");
    } catch (const MpsError& fixed_err) {
      error = "free format: " + free_err.what + " | fixed format: " + fixed_err.what;
      return false;
    }
  }
  if (auto err = M.validate(); !err.empty()) {
    error = "invalid model: " + err;
    return false;
  }
  return true;
}

bool read_mps(const std::string& path, Model& M, ModelInfo& info, std::string& error) {
  if (path.size() >= 3 && path.compare(path.size() - 3, 3, ".gz") == 0) {
    error = "gzip-compressed input is not supported; decompress the file first";
    return false;
  }
  std::string text;
  return slurp(path, text, error) && read_mps_text(text, M, info, error);
}

bool read_model(const std::string& path, Model& M, ModelInfo& info, std::string& error) {
  auto ends = [&](const char* suf) {
    const std::size_t n = std::char_traits<char>::length(suf);
    return path.size() >= n && path.compare(path.size() - n, n, suf) == 0;
  };
  if (ends(".lpm")) return read_lpm(path, M, info, error);
  if (ends(".mps") || ends(".MPS")) return read_mps(path, M, info, error);
  error = "unknown file type (expected .mps or .lpm)";
  return false;
}

// ------------------------------------------------------------------------------- .sol
bool write_solution(const std::string& path, const Model& m, const ModelInfo& info, const Solution& s,
                    std::string& error) {
  std::FILE* f = std::fopen(path.c_str(), "w");
  if (!f) {
    error = "cannot open " + path + " for writing";
    return false;
  }
  std::fprintf(f, "PS26119-SOLUTION 1\n");
  std::fprintf(f, "model %s\n", s.model_fingerprint.empty() ? fingerprint_hex(m).c_str() : s.model_fingerprint.c_str());
  std::fprintf(f, "name %s\n", info.name.c_str());
  std::fprintf(f, "status %s\n", status_name(s.status));
  std::fprintf(f, "engine %s\n", s.engine.c_str());
  std::fprintf(f, "precision %s\n", s.precision.c_str());
  std::fprintf(f, "objective %.17g\n", s.objective);
  std::fprintf(f, "dual_objective %.17g\n", s.dual_objective);
  if (s.certified_bound == s.certified_bound) std::fprintf(f, "certified_bound %.17g\n", s.certified_bound);
  std::fprintf(f, "primal_residual %.6g\n", s.primal_residual);
  std::fprintf(f, "dual_residual %.6g\n", s.dual_residual);
  std::fprintf(f, "gap %.6g\n", s.gap);
  std::fprintf(f, "iterations %lld\n", s.iterations);
  std::fprintf(f, "seconds %.6f\n", s.seconds);
  std::fprintf(f, "setup_seconds %.6f\n", s.setup_seconds);
  if (s.primal_weight == s.primal_weight) std::fprintf(f, "primal_weight %.17g\n", s.primal_weight);
  if (s.iterations_to_fast >= 0) std::fprintf(f, "iterations_to_fast %lld\n", s.iterations_to_fast);
  if (!s.check.empty())
    std::fprintf(f, "check %s primal %.3g dual %.3g gap %.3g\n", s.check.c_str(), s.check_primal, s.check_dual,
                 s.check_gap);
  if (!s.message.empty()) std::fprintf(f, "message %s\n", s.message.c_str());
  const bool primal = static_cast<int>(s.x.size()) == m.num_cols;
  const bool dual = static_cast<int>(s.z.size()) == m.num_cols && static_cast<int>(s.y.size()) == m.num_rows;
  if (primal) {
    std::fprintf(f, "COLUMNS %d\n", m.num_cols);
    for (int j = 0; j < m.num_cols; ++j)
      std::fprintf(f, "%d %.17g %.17g %s\n", j, s.x[j], dual ? s.z[j] : 0.0,
                   j < static_cast<int>(info.col_names.size()) ? info.col_names[j].c_str() : "");
    std::fprintf(f, "ROWS %d\n", m.num_rows);
    const std::vector<double> act = m.row_activity(s.x);
    for (int i = 0; i < m.num_rows; ++i)
      std::fprintf(f, "%d %.17g %.17g %s\n", i, act[i], dual ? s.y[i] : 0.0,
                   i < static_cast<int>(info.row_names.size()) ? info.row_names[i].c_str() : "");
  }
  auto ray = [&](const char* key, const std::vector<double>& v) {
    if (v.empty()) return;
    std::fprintf(f, "%s %zu\n", key, v.size());
    for (std::size_t k = 0; k < v.size(); ++k) std::fprintf(f, "%zu %.17g\n", k, v[k]);
  };
  ray("DUAL_RAY", s.dual_ray);
  ray("PRIMAL_RAY", s.primal_ray);
  std::fprintf(f, "END\n");
  const bool ok = std::fclose(f) == 0;
  if (!ok) error = "write failed for " + path;
  return ok;
}

}  // namespace b200
