// Matrix Market reader with the interface the reference's converters use
// (matrix_market::reader / matrix_class / matrix_meta, consumed at
// common/matrix_converter.cpp:15-33 and common/scoo_matrix_class.h:25; the
// reference's own reader is an external submodule that is not vendored).
//
// Reads "%%MatrixMarket matrix coordinate <real|integer|pattern>
// <general|symmetric|skew-symmetric>" files.  Symmetric and skew-symmetric
// matrices are expanded to general on reading (the mirrored off-diagonal
// entries are appended, negated for skew-symmetric), so the converters, which
// accept only general storage, take every supported file.  Pattern entries
// get the value 1.  Indices in the file are 1-based; the reader stores them
// 0-based.  Malformed input throws std::runtime_error.
#pragma once

#include <cstdint>
#include <istream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace matrix_market {

class matrix_class {
 public:
  enum class storage_scheme { general = 0, symmetric = 1, skew_symmetric = 2 };
  struct matrix_meta {
    unsigned int rows_count = 0;
    unsigned int cols_count = 0;
    unsigned int non_zero_count = 0;
    storage_scheme matrix_storage_scheme = storage_scheme::general;
  };
  matrix_meta meta;

  const unsigned int *get_row_ids() const { return row_ids.data(); }
  const unsigned int *get_col_ids() const { return col_ids.data(); }
  const double *get_dbl_data() const { return values.data(); }

  std::vector<unsigned int> row_ids, col_ids;
  std::vector<double> values;
};

class reader {
 public:
  explicit reader(std::istream &is) { parse(is); }
  const matrix_class &matrix() const { return m_; }

 private:
  static std::string lower(std::string s) {
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
  }

  void parse(std::istream &is) {
    std::string line;
    if (!std::getline(is, line)) throw std::runtime_error("matrix market: empty input");
    std::istringstream h(line);
    std::string banner, object, format, field, symmetry;
    h >> banner >> object >> format >> field >> symmetry;
    if (lower(banner) != "%%matrixmarket" || lower(object) != "matrix")
      throw std::runtime_error("matrix market: bad banner '" + line + "'");
    if (lower(format) != "coordinate") throw std::runtime_error("matrix market: only coordinate format is supported");
    field = lower(field);
    symmetry = lower(symmetry);
    const bool pattern = field == "pattern";
    if (!pattern && field != "real" && field != "integer" && field != "double")
      throw std::runtime_error("matrix market: unsupported field '" + field + "'");
    int sym = 0;
    if (symmetry == "symmetric") sym = 1;
    else if (symmetry == "skew-symmetric") sym = 2;
    else if (symmetry != "general") throw std::runtime_error("matrix market: unsupported symmetry '" + symmetry + "'");

    while (std::getline(is, line))
      if (!line.empty() && line[0] != '%') break;
    std::istringstream sz(line);
    unsigned long long rows = 0, cols = 0, entries = 0;
    if (!(sz >> rows >> cols >> entries)) throw std::runtime_error("matrix market: bad size line '" + line + "'");
    if (rows > UINT32_MAX || cols > UINT32_MAX || entries > UINT32_MAX)
      throw std::runtime_error("matrix market: sizes exceed 32-bit indexing");
    m_.row_ids.reserve(entries * (sym ? 2 : 1));
    m_.col_ids.reserve(entries * (sym ? 2 : 1));
    m_.values.reserve(entries * (sym ? 2 : 1));
    for (unsigned long long k = 0; k < entries; ++k) {
      unsigned long long r = 0, c = 0;
      double v = 1.0;
      if (!(is >> r >> c)) throw std::runtime_error("matrix market: truncated entry list");
      if (!pattern && !(is >> v)) throw std::runtime_error("matrix market: missing value");
      if (r < 1 || c < 1 || r > rows || c > cols) throw std::runtime_error("matrix market: index out of range");
      push(r - 1, c - 1, v);
      if (sym && r != c) push(c - 1, r - 1, sym == 2 ? -v : v);
    }
    m_.meta.rows_count = (unsigned)rows;
    m_.meta.cols_count = (unsigned)cols;
    if (m_.values.size() > UINT32_MAX) throw std::runtime_error("matrix market: expanded entries exceed 32-bit indexing");
    m_.meta.non_zero_count = (unsigned)m_.values.size();
    m_.meta.matrix_storage_scheme = matrix_class::storage_scheme::general;
  }
  void push(unsigned long long r, unsigned long long c, double v) {
    m_.row_ids.push_back((unsigned)r);
    m_.col_ids.push_back((unsigned)c);
    m_.values.push_back(v);
  }

  matrix_class m_;
};

}  // namespace matrix_market
