// Builds the C++ host-layer classes (matrix_market::reader, csr/ell/coo/
// hybrid_matrix_class, scoo_matrix_class, get_rows_statistics) from a Matrix
// Market file, in float and double, and writes every array as raw binary
// <out>/<name>_<f32|f64>.bin for the Python test to compare with the fixtures
// the reference's own sources produced.
//
//     host_classes_check file.mtx outdir
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>

#include "matrix_converter.h"
#include "matrix_market_reader.h"
#include "scoo_matrix_class.h"

static std::string out_dir;

template <typename T>
static void dump(const std::string &name, const T *p, size_t n) {
  std::ofstream os(out_dir + "/" + name + ".bin", std::ios::binary);
  if (n) os.write(reinterpret_cast<const char *>(p), n * sizeof(T));
}

template <typename T>
static void run(const matrix_market::matrix_class &mm, const std::string &s) {
  csr_matrix_class<T> csr(mm);
  const auto &meta = csr.meta;
  dump("csr_row_ptr_" + s, csr.row_ptr.get(), meta.rows_count + 1);
  dump("csr_columns_" + s, csr.columns.get(), meta.non_zero_count);
  dump("csr_data_" + s, csr.data.get(), meta.non_zero_count);
  const auto st = get_rows_statistics(meta, csr.row_ptr.get());
  const unsigned stats[3] = {st.min_elements_in_rows, st.max_elements_in_rows, st.avg_elements_in_rows};
  dump("stats_u32_" + s, stats, 3);
  dump("stats_std_" + s, &st.elements_in_rows_std_deviation, 1);
  const unsigned ell_est = (unsigned)ell_matrix_class<T>::estimate_size(csr);
  dump("ell_estimate_" + s, &ell_est, 1);
  if (ell_est <= (1u << 22)) {
    ell_matrix_class<T> ell(csr);
    dump("ell_width_" + s, &ell.elements_in_rows, 1);
    dump("ell_data_" + s, ell.data.get(), ell.get_matrix_size());
    dump("ell_columns_" + s, ell.columns.get(), ell.get_matrix_size());
  }
  coo_matrix_class<T> coo(csr);
  dump("coo_data_" + s, coo.data.get(), coo.get_matrix_size());
  dump("coo_cols_" + s, coo.cols.get(), coo.get_matrix_size());
  dump("coo_rows_" + s, coo.rows.get(), coo.get_matrix_size());
  hybrid_matrix_class<T> hyb(csr);
  hyb.allocate(csr, 0.2);
  dump("hyb_width_" + s, &hyb.ell_matrix->elements_in_rows, 1);
  dump("hyb_ell_data_" + s, hyb.ell_matrix->data.get(), hyb.ell_matrix->get_matrix_size());
  dump("hyb_ell_columns_" + s, hyb.ell_matrix->columns.get(), hyb.ell_matrix->get_matrix_size());
  dump("hyb_coo_data_" + s, hyb.coo_matrix->data.get(), hyb.coo_matrix->get_matrix_size());
  dump("hyb_coo_cols_" + s, hyb.coo_matrix->cols.get(), hyb.coo_matrix->get_matrix_size());
  dump("hyb_coo_rows_" + s, hyb.coo_matrix->rows.get(), hyb.coo_matrix->get_matrix_size());
  for (auto [tag, sm, smem] : {std::make_tuple("scoo", 148u, (size_t)49152), std::make_tuple("scoo_small", 4u, (size_t)1024)}) {
    scoo_matrix_class<T> sc(sm, smem, csr);
    const unsigned prm[3] = {sc.slices_count, sc.slice_size, sc.lane_size};
    const std::string t(tag);
    dump(t + "_params_" + s, prm, 3);
    dump(t + "_values_" + s, sc.values.get(), sc.get_matrix_size());
    dump(t + "_c_index_" + s, sc.c_index.get(), sc.get_matrix_size());
    dump(t + "_r_index_" + s, sc.r_index.get(), sc.get_matrix_size());
    dump(t + "_slices_ptr_" + s, sc.slices_ptr.get(), sc.slices_count + 1);
  }
}

int main(int argc, char **argv) {
  if (argc != 3) {
    std::cerr << "usage: host_classes_check file.mtx outdir" << std::endl;
    return 1;
  }
  out_dir = argv[2];
  try {
    std::ifstream is(argv[1]);
    matrix_market::reader reader(is);
    run<float>(reader.matrix(), "f32");
    run<double>(reader.matrix(), "f64");
  } catch (const std::exception &e) {
    std::cerr << "error: " << e.what() << std::endl;
    return 2;
  }
  return 0;
}
