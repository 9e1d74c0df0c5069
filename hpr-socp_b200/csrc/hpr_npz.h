// hpr_npz.h — streaming writer of NumPy .npz archives (a ZIP of .npy members,
// stored without compression).
//
// The solver's auto-save checkpoint is written in this container: every
// array and scalar of the reference's HDF5 auto-save file
// (save_state_to_hdf5!, src/algorithm.jl:306-421) becomes one member whose
// name is the HDF5 path ("current/x_org", "best/sigma", ...).  NumPy reads
// it with np.load, Julia with NPZ.jl.
//
// Members are written as they are added (the CRC-32 is computed over the
// member's bytes first), so no archive-sized buffer is held.  ZIP64 records
// are written for members and directories that pass 4 GiB, or for every
// member when `force_zip64` is set.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace hpr {

// CRC-32 (ISO-HDLC polynomial 0xEDB88320, the checksum of ZIP members),
// continued from `crc` (0 for a fresh checksum).
uint32_t crc32_update(uint32_t crc, const void* data, size_t bytes);

class NpzWriter {
 public:
  explicit NpzWriter(bool force_zip64 = false) : force_zip64_(force_zip64) {}
  ~NpzWriter();
  NpzWriter(const NpzWriter&) = delete;
  NpzWriter& operator=(const NpzWriter&) = delete;

  bool open(const std::string& path);
  // One .npy member: `descr` is the NumPy type string ("<f8", "<i8", "|b1",
  // "<U12"), `shape` empty for a 0-d array, `data` the C-ordered elements.
  // `crc`, when given, is member_crc() of the same arguments (computed
  // beforehand, for example on another thread).
  bool add_array(const std::string& name, const std::string& descr, const std::vector<int64_t>& shape,
                 const void* data, size_t bytes, const uint32_t* crc = nullptr);
  // The .npy header of a member, and the CRC-32 of header and data.
  static std::string npy_header(const std::string& descr, const std::vector<int64_t>& shape);
  static uint32_t member_crc(const std::string& descr, const std::vector<int64_t>& shape, const void* data,
                             size_t bytes);
  bool add_f64(const std::string& name, double v);
  bool add_i64(const std::string& name, int64_t v);
  bool add_bool(const std::string& name, bool v);
  bool add_string(const std::string& name, const std::string& s);  // ASCII -> '<U{len}'
  bool add_vector(const std::string& name, const double* v, int64_t n, const uint32_t* crc = nullptr);
  // Writes the central directory and closes the file.
  bool close();
  const std::string& error() const { return err_; }

 private:
  struct Entry {
    std::string name;
    uint32_t crc;
    uint64_t size;
    uint64_t offset;
    bool zip64;
  };
  bool put(const void* p, size_t n);
  bool fail(const std::string& msg);
  bool force_zip64_;
  FILE* f_ = nullptr;
  uint64_t pos_ = 0;
  uint16_t dos_time_ = 0, dos_date_ = 0;
  std::vector<Entry> entries_;
  std::string err_;
};

}  // namespace hpr
