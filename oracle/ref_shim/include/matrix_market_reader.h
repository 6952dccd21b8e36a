// Stand-in for the reference's external/matrix_reader submodule (absent from
// the reference checkout).  Provides only what common/matrix_converter.cpp,
// common/scoo_matrix_class.cpp and gpu/csr_adaptive_spmv.cu use:
// matrix_class::meta {rows_count, cols_count, non_zero_count,
// matrix_storage_scheme}, storage_scheme::general and the three COO accessors
// (uses at matrix_converter.cpp:17-33).  Test infrastructure only.
#ifndef MFP_ORACLE_MATRIX_MARKET_READER_H
#define MFP_ORACLE_MATRIX_MARKET_READER_H

#include <vector>

namespace matrix_market {

class matrix_class {
public:
  enum class storage_scheme { general, symmetric, skew_symmetric, hermitian };

  struct matrix_meta {
    unsigned int rows_count = 0;
    unsigned int cols_count = 0;
    unsigned int non_zero_count = 0;
    storage_scheme matrix_storage_scheme = storage_scheme::general;
  };

  matrix_meta meta;
  std::vector<unsigned int> row_ids, col_ids;
  std::vector<double> values;

  const unsigned int *get_row_ids() const { return row_ids.data(); }
  const unsigned int *get_col_ids() const { return col_ids.data(); }
  const double *get_dbl_data() const { return values.data(); }
};

}  // namespace matrix_market

#endif
