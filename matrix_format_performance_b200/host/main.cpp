// Benchmark driver with the reference's command line and result files
// (main.cpp:82-283 perform_measurement, :395-505 main):
//
//     mfp_driver [--hybrid-sweep] /path/to/mtx_list
//
// For every Matrix Market file named in the list (one path per line), in
// float and double: CSR conversion, the CPU CSR columns (one single-thread run
// as the reference answer, 20 parallel runs), then 20 runs of every GPU
// operator (CSR, CSR vector, CSR-Adaptive, the cuSPARSE CSR yardstick, ELL,
// COO, SCOO, hybrid with the reference's 0.2 split, under both hybrid
// labels), averaged by
// measurement_class.  Results go to the reference's files in the working
// directory: float.json / double.json (seconds), *_effective_bandwidth.json,
// *_computational_throughput.json ([matrix file name][label]), and
// matrices_info.json (nnz, rows, cols).  Extra, for the engine:
// *_model_bandwidth.json (the algorithmic byte model per label) and
// *_max_error.json (largest compare_results error per label).
//
// Matrices that do not fit in 90% of the free device memory (CSR or ELL
// layout plus five vectors, as the reference estimates) are skipped, as are
// ELL layouts more than 64x larger than the CSR layout (the engine measures
// the other formats of such a matrix rather than dropping it).
// --hybrid-sweep adds the reference's disabled hybrid sweep (main.cpp:247-279):
// ELL part from avg + (max - avg) * percent for percent = 0, 0.35, 0.70, both
// hybrid operators, 20 runs each, keyed "<label> <percent>%" (the reference's
// per-percent labels are commented out, so its results would collide); a
// percent whose ELL part is more than 64x the CSR layout is skipped.
// Clocks are never changed: the reference's application-clock locking is not
// built.  MKL and cusp columns are not measured.
#include <cuda_runtime.h>

#include <cstdio>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "cpu_matrix_multiplier.h"
#include "cusparse_yardstick.h"
#include "gpu_matrix_multiplier.h"
#include "matrix_converter.h"
#include "matrix_market_reader.h"
#include "measurement_class.h"
#include "resizable_gpu_memory.h"
#include "scoo_matrix_class.h"

namespace {

using table = std::map<std::string, std::map<std::string, double>>;  // [matrix][label]

std::string json_escape(const std::string &s) {
  std::string o;
  for (char c : s) {
    if (c == '"' || c == '\\') o += '\\';
    o += c;
  }
  return o;
}

void write_json(const std::string &path, const table &t) {
  std::ofstream os(path);
  os.precision(17);
  os << "{";
  bool first_m = true;
  for (auto &[mtx, row] : t) {
    os << (first_m ? "\n" : ",\n") << "  \"" << json_escape(mtx) << "\": {";
    first_m = false;
    bool first = true;
    for (auto &[label, v] : row) {
      os << (first ? "\n" : ",\n") << "    \"" << json_escape(label) << "\": " << v;
      first = false;
    }
    os << "\n  }";
  }
  os << "\n}\n";
}

std::string file_name(const std::string &path) {
  const size_t i = path.rfind('/');
  return i == std::string::npos ? path : path.substr(i + 1);
}

template <typename data_type>
std::vector<measurement_class> perform_measurement(const matrix_market::reader &reader, size_t free_memory,
                                                   int sm_count, size_t shared_mem_size, bool hybrid_sweep) {
  std::vector<measurement_class> out;
  csr_matrix_class<data_type> csr(reader.matrix());
  const auto &meta = csr.meta;
  const size_t vec = (size_t)std::max(meta.rows_count, meta.cols_count) * sizeof(data_type);
  const size_t csr_bytes = csr.get_matrix_size() * (sizeof(data_type) + 4);
  const size_t ell_bytes = ell_matrix_class<data_type>::estimate_size(csr) * (sizeof(data_type) + 4);
  if (std::max(csr_bytes, std::min(ell_bytes, 64 * csr_bytes)) + 5 * vec > free_memory * 0.9) return {};
  const bool with_ell = ell_bytes <= 64 * std::max<size_t>(csr_bytes, 1);

  std::unique_ptr<data_type[]> reference_answer(new data_type[std::max(1u, meta.rows_count)]);
  std::unique_ptr<data_type[]> reduce_order_answer(new data_type[std::max(1u, meta.rows_count)]);
  std::unique_ptr<data_type[]> cpu_y(new data_type[std::max(1u, meta.rows_count)]);
  std::unique_ptr<data_type[]> x(new data_type[std::max(1u, std::max(meta.rows_count, meta.cols_count))]);

  out.push_back(cpu_csr_spmv_single_thread_naive(csr, x.get(), reference_answer.get()));
  auto repeat = [&](const std::function<measurement_class(bool)> &action) {
    measurement_class r;
    for (unsigned i = 0; i < 20; ++i) r += action(i == 0);
    r.finalize();
    out.push_back(r);
    std::cout << "  " << r.get_format() << ": " << r.get_elapsed() * 1e3 << " ms, " << r.get_model_bandwidth()
              << " GB/s (model)" << std::endl;
  };
  repeat([&](bool) { return cpu_csr_spmv_multi_thread_naive(csr, x.get(), cpu_y.get()); });
  cpu_csr_spmv_single_thread_naive_with_reduce_order(csr, x.get(), reduce_order_answer.get());

  resizable_gpu_memory<data_type> A, x_gpu, y, A_coo;
  resizable_gpu_memory<unsigned int> col_ids, row_ptr, col_ids_coo;
  repeat([&](bool) { return gpu_csr_spmv<data_type>(csr, A, col_ids, row_ptr, x_gpu, y, x.get(), reference_answer.get()); });
  repeat([&](bool) {
    return gpu_csr_vector_spmv<data_type>(csr, A, col_ids, row_ptr, x_gpu, y, x.get(), reduce_order_answer.get());
  });
  repeat([&](bool) {
    return gpu_csr_adaptive_spmv<data_type>(csr, A, col_ids, row_ptr, x_gpu, y, x.get(), reference_answer.get());
  });
  repeat([&](bool) {
    return gpu_csr_cusparse_spmv<data_type>(csr, A, col_ids, row_ptr, x_gpu, y, x.get(), reference_answer.get());
  });
  if (with_ell) {
    ell_matrix_class<data_type> ell(csr);
    repeat([&](bool) { return gpu_ell_spmv<data_type>(ell, A, col_ids, x_gpu, y, x.get(), reference_answer.get()); });
  }
  {
    coo_matrix_class<data_type> coo(csr);
    repeat([&](bool) {
      return gpu_coo_spmv<data_type>(coo, A, col_ids, row_ptr, x_gpu, y, x.get(), reference_answer.get());
    });
  }
  {
    scoo_matrix_class<data_type> scoo(sm_count, shared_mem_size, csr);
    std::cout << "  SCOO: slice_size=" << scoo.slice_size << "; lane_size=" << scoo.lane_size
              << "; slices_count=" << scoo.slices_count << std::endl;
    repeat([&](bool print_diff) {
      return gpu_scoo_spmv<data_type>(print_diff, scoo, A, col_ids, row_ptr, x_gpu, y, x.get(), reference_answer.get());
    });
  }
  {
    hybrid_matrix_class<data_type> hybrid(csr);
    hybrid.allocate(csr, 0.2);
    repeat([&](bool) {
      return gpu_hybrid_spmv<data_type>(hybrid, A, A_coo, col_ids, col_ids_coo, row_ptr, x_gpu, y, x.get(),
                                        reference_answer.get());
    });
    repeat([&](bool) {
      return gpu_hybrid_atomic_spmv<data_type>(hybrid, A, A_coo, col_ids, col_ids_coo, row_ptr, x_gpu, y, x.get(),
                                               reference_answer.get());
    });
  }
  if (hybrid_sweep) {
    const auto st = get_rows_statistics(meta, csr.row_ptr.get());
    hybrid_matrix_class<data_type> hybrid(csr);
    for (int step = 0; step < 3; ++step) {
      const double percent = 0.35 * step;  // the reference's loop: 0.0, 0.35, 0.70 (<= 1.0)
      const unsigned int width = st.avg_elements_in_rows + (st.max_elements_in_rows - st.avg_elements_in_rows) * percent;
      if ((size_t)width * meta.rows_count * (sizeof(data_type) + 4) > 64 * std::max<size_t>(csr_bytes, 1)) continue;
      hybrid.allocate(csr, percent);
      const std::string tag = " " + std::to_string((int)(percent * 100)) + "%";
      repeat([&](bool) {
        auto m = gpu_hybrid_spmv<data_type>(hybrid, A, A_coo, col_ids, col_ids_coo, row_ptr, x_gpu, y, x.get(),
                                            reference_answer.get());
        m.set_format(m.get_format() + tag);
        return m;
      });
      repeat([&](bool) {
        auto m = gpu_hybrid_atomic_spmv<data_type>(hybrid, A, A_coo, col_ids, col_ids_coo, row_ptr, x_gpu, y, x.get(),
                                                   reference_answer.get());
        m.set_format(m.get_format() + tag);
        return m;
      });
    }
  }
  return out;
}

}  // namespace

int main(int argc, char *argv[]) {
  const bool hybrid_sweep = argc == 3 && std::string(argv[1]) == "--hybrid-sweep";
  if (argc != 2 && !hybrid_sweep) {
    std::cerr << "Usage: " << argv[0] << " [--hybrid-sweep] /path/to/mtx_list" << std::endl;
    return 1;
  }
  const char *list_path = argv[argc - 1];
  const int gpu_id = 0;
  if (cudaSetDevice(gpu_id) != cudaSuccess) {
    std::cerr << "CUDA device " << gpu_id << " is not available" << std::endl;
    return 1;
  }
  mfp_device_info dev{};
  if (mfp_get_device_info(gpu_id, &dev) != MFP_SUCCESS) {
    std::cerr << "mfp_get_device_info: " << mfp_last_error() << std::endl;
    return 1;
  }
  size_t free_mem = 0, total_mem = 0;
  if (cudaMemGetInfo(&free_mem, &total_mem) != cudaSuccess) {
    std::cerr << "CUDA Can't get free memory!" << std::endl;
    return 1;
  }

  std::ifstream list(list_path);
  if (!list) {
    std::cerr << "cannot open " << list_path << std::endl;
    return 1;
  }
  std::map<std::string, table> elapsed, bandwidth, throughput, model_bw, max_error;
  std::map<std::string, std::map<std::string, double>> info;
  std::string mtx;
  int status = 0;
  while (std::getline(list, mtx)) {
    if (mtx.empty()) continue;
    try {
      std::cout << "Start loading matrix " << mtx << std::endl;
      std::ifstream is(mtx);
      if (!is) throw std::runtime_error("cannot open " + mtx);
      matrix_market::reader reader(is);
      const auto &meta = reader.matrix().meta;
      std::cout << "Complete loading (rows: " << meta.rows_count << "; cols: " << meta.cols_count
                << "; nnz: " << meta.non_zero_count << ")" << std::endl;
      std::map<std::string, std::vector<measurement_class>> results;
      results["float"] =
          perform_measurement<float>(reader, free_mem, dev.sm_count, dev.shared_mem_per_block, hybrid_sweep);
      results["double"] =
          perform_measurement<double>(reader, free_mem, dev.sm_count, dev.shared_mem_per_block, hybrid_sweep);
      const std::string name = file_name(mtx);
      if (results["float"].empty() || results["double"].empty()) continue;  // did not fit on the GPU
      for (auto &[type, res] : results)
        for (auto &m : res) {
          elapsed[type][name][m.get_format()] = m.get_elapsed();
          bandwidth[type][name][m.get_format()] = m.get_effective_bandwidth();
          throughput[type][name][m.get_format()] = m.get_computational_throughput();
          model_bw[type][name][m.get_format()] = m.get_model_bandwidth();
          max_error[type][name][m.get_format()] = m.error;
        }
      info[name]["nnz"] = meta.non_zero_count;
      info[name]["rows"] = meta.rows_count;
      info[name]["cols"] = meta.cols_count;
    } catch (const std::exception &e) {
      std::cerr << "matrix " << mtx << ": " << e.what() << std::endl;
      status = 2;
    }
  }
  write_json("matrices_info.json", info);
  for (const char *p : {"float", "double"}) {
    const std::string s(p);
    write_json(s + ".json", elapsed[s]);
    write_json(s + "_effective_bandwidth.json", bandwidth[s]);
    write_json(s + "_computational_throughput.json", throughput[s]);
    write_json(s + "_model_bandwidth.json", model_bw[s]);
    write_json(s + "_max_error.json", max_error[s]);
  }
  return status;
}
