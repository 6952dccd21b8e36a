// measurement_class and compare_results with the reference's interface
// (common/measurement_class.h:11-89, measurement_class.cpp:7-16): a label,
// elapsed seconds, effective bandwidth = load/store bytes / (elapsed * 1e9) and
// computational throughput = operations / (elapsed * 1e9); += and finalize()
// average repeated measurements.  The reference's per-format byte counts are
// kept for comparable JSON; model_bandwidth() adds the format-independent
// algorithmic model nnz*(sizeof(T)+4) + (rows+1)*4 + cols*sizeof(T) +
// rows*sizeof(T) divided by the same time.
#pragma once

#include <cmath>
#include <iostream>
#include <string>
#include <utility>

class measurement_class {
  static constexpr double giga = 1e9;

 public:
  measurement_class() = default;
  measurement_class(std::string format, double elapsed_arg, double load_store_bytes, double operations_count,
                    double model_bytes = 0.0)
      : elapsed(elapsed_arg),
        effective_bandwidth(load_store_bytes / (elapsed_arg * giga)),
        computational_throughput(operations_count / (elapsed_arg * giga)),
        model_bandwidth_(model_bytes / (elapsed_arg * giga)),
        matrix_format(std::move(format)) {}

  double get_elapsed() const { return elapsed; }
  double get_effective_bandwidth() const { return effective_bandwidth; }
  double get_computational_throughput() const { return computational_throughput; }
  double get_model_bandwidth() const { return model_bandwidth_; }
  const std::string &get_format() const { return matrix_format; }
  // engine extension: relabel a record (the hybrid sweep keys its results by percent)
  void set_format(std::string f) { matrix_format = std::move(f); }
  // relative squared L2 error of the last compare_results against the reference answer
  double error = 0.0;

  measurement_class &operator+=(const measurement_class &rhs) {
    elapsed += rhs.get_elapsed();
    effective_bandwidth += rhs.get_effective_bandwidth();
    computational_throughput += rhs.get_computational_throughput();
    model_bandwidth_ += rhs.get_model_bandwidth();
    error = std::max(error, rhs.error);
    matrix_format = rhs.get_format();
    measurements_count++;
    return *this;
  }

  void finalize() {
    if (measurements_count) {
      elapsed /= measurements_count;
      effective_bandwidth /= measurements_count;
      computational_throughput /= measurements_count;
      model_bandwidth_ /= measurements_count;
    }
  }

 private:
  double elapsed = 0.0;
  double effective_bandwidth = 0.0;
  double computational_throughput = 0.0;
  double model_bandwidth_ = 0.0;
  std::string matrix_format;
  unsigned int measurements_count = 0;
};

// Relative squared L2 error sum (a-b)^2 / sum b^2, accumulated in data_type.
// Above 1e-9 it reports the error and the first element off by more than 1e-8
// on stderr (the reference's behaviour) and returns the error.
template <typename data_type>
double compare_results(unsigned int y_size, const data_type *a, const data_type *b) {
  data_type numerator = 0, denominator = 0;
  for (unsigned int i = 0; i < y_size; i++) {
    numerator += (a[i] - b[i]) * (a[i] - b[i]);
    denominator += b[i] * b[i];
  }
  const data_type error = numerator / denominator;
  if (error > 1e-9) {
    std::cerr << "ERROR: " << error << std::endl;
    for (unsigned int i = 0; i < y_size; i++)
      if (std::abs(a[i] - b[i]) > 1e-8) {
        std::cerr << "a[" << i << "] = " << a[i] << "; b[" << i << "] = " << b[i] << std::endl;
        break;
      }
  }
  std::cerr.flush();
  return (double)error;
}
