// Drives the library's .npz writer (hpr-socp_b200/csrc/hpr_npz.cpp) for
// tests/test_npz.py: writes one archive with every member type, plain or
// with forced ZIP64 records, and prints CRC-32 values of fixed inputs.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../hpr-socp_b200/csrc/hpr_npz.h"

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const std::string path = argv[1];
  const bool zip64 = std::atoi(argv[2]) != 0;
  hpr::NpzWriter w(zip64);
  std::vector<double> v(100003);
  for (size_t i = 0; i < v.size(); ++i) v[i] = 0.5 * (double)i - 3.25;
  const int64_t mat_shape0 = 3, mat_shape1 = 4;
  std::vector<int64_t> mat(mat_shape0 * mat_shape1);
  for (size_t i = 0; i < mat.size(); ++i) mat[i] = (int64_t)i * 7 - 20;
  bool ok = w.open(path) && w.add_vector("current/x_org", v.data(), (int64_t)v.size()) &&
            w.add_vector("best/y_org", v.data(), 0) && w.add_f64("current/sigma", 1.25) &&
            w.add_i64("best/iteration", 150) && w.add_bool("parameters/auto_save", true) &&
            w.add_bool("parameters/use_l2_scaling", false) &&
            w.add_string("current/timestamp", "2026-01-02T03:04:05.678") && w.add_string("empty", "") &&
            w.add_array("matrix", "<i8", {mat_shape0, mat_shape1}, mat.data(), mat.size() * sizeof(int64_t));
  ok = w.close() && ok;
  if (!ok) {
    std::printf("error %s\n", w.error().c_str());
    return 1;
  }
  // CRC-32 of fixed inputs, each length 0..40, split at every point
  std::string bytes;
  for (int i = 0; i < 40; ++i) bytes.push_back((char)(i * 37 + 11));
  for (size_t len = 0; len <= bytes.size(); ++len) {
    const uint32_t whole = hpr::crc32_update(0, bytes.data(), len);
    for (size_t cut = 0; cut <= len; ++cut) {
      const uint32_t split = hpr::crc32_update(hpr::crc32_update(0, bytes.data(), cut), bytes.data() + cut, len - cut);
      if (split != whole) {
        std::printf("split mismatch %zu %zu\n", len, cut);
        return 1;
      }
    }
    std::printf("crc %zu %u\n", len, whole);
  }
  return 0;
}
