// hpr_npz.cpp — streaming .npz writer (see hpr_npz.h).
//
// Layouts written here are the published ones: the .npy format (NumPy
// Enhancement Proposal 1, version 1.0 headers padded to 64 bytes) and the
// ZIP local header / central directory / end record, with the ZIP64 extra
// field (tag 0x0001) and ZIP64 end record and locator (PKWARE APPNOTE 4.5).
#include "hpr_npz.h"

#include <ctime>

namespace hpr {

namespace {

// slicing-by-8 tables of the reflected CRC-32
struct Crc32Tables {
  uint32_t t[8][256];
  Crc32Tables() {
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for (int k = 0; k < 8; ++k) c = (c & 1u) ? (c >> 1) ^ 0xEDB88320u : (c >> 1);
      t[0][i] = c;
    }
    for (uint32_t i = 0; i < 256; ++i)
      for (int s = 1; s < 8; ++s) t[s][i] = (t[s - 1][i] >> 8) ^ t[0][t[s - 1][i] & 0xFFu];
  }
};
const Crc32Tables& crc_tables() {
  static const Crc32Tables tables;
  return tables;
}

inline uint32_t load_le32(const unsigned char* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

constexpr uint64_t k32Max = 0xFFFFFFFFull;

std::string shape_string(const std::vector<int64_t>& shape) {
  if (shape.empty()) return "()";
  std::string s = "(";
  for (size_t i = 0; i < shape.size(); ++i) {
    if (i) s += ", ";
    s += std::to_string(shape[i]);
  }
  if (shape.size() == 1) s += ",";
  return s + ")";
}

}  // namespace

uint32_t crc32_update(uint32_t crc, const void* data, size_t bytes) {
  const auto& T = crc_tables().t;
  const unsigned char* p = static_cast<const unsigned char*>(data);
  uint32_t c = ~crc;
  while (bytes >= 8) {
    const uint32_t a = load_le32(p) ^ c, b = load_le32(p + 4);
    c = T[7][a & 0xFFu] ^ T[6][(a >> 8) & 0xFFu] ^ T[5][(a >> 16) & 0xFFu] ^ T[4][a >> 24] ^ T[3][b & 0xFFu] ^
        T[2][(b >> 8) & 0xFFu] ^ T[1][(b >> 16) & 0xFFu] ^ T[0][b >> 24];
    p += 8;
    bytes -= 8;
  }
  while (bytes--) c = T[0][(c ^ *p++) & 0xFFu] ^ (c >> 8);
  return ~c;
}

NpzWriter::~NpzWriter() {
  if (f_) std::fclose(f_);
}

bool NpzWriter::fail(const std::string& msg) {
  if (err_.empty()) err_ = msg;
  return false;
}

bool NpzWriter::put(const void* p, size_t n) {
  if (!f_) return fail("archive is not open");
  if (n && std::fwrite(p, 1, n, f_) != n) return fail("write failed");
  pos_ += n;
  return true;
}

bool NpzWriter::open(const std::string& path) {
  f_ = std::fopen(path.c_str(), "wb");
  if (!f_) return fail("cannot open " + path + " for writing");
  std::setvbuf(f_, nullptr, _IOFBF, 1 << 20);
  std::time_t now = std::time(nullptr);
  std::tm tmv{};
  localtime_r(&now, &tmv);
  const int year = tmv.tm_year + 1900 < 1980 ? 1980 : tmv.tm_year + 1900;
  dos_time_ = (uint16_t)((tmv.tm_hour << 11) | (tmv.tm_min << 5) | (tmv.tm_sec / 2));
  dos_date_ = (uint16_t)(((year - 1980) << 9) | ((tmv.tm_mon + 1) << 5) | tmv.tm_mday);
  return true;
}

// .npy header: magic, version 1.0, little-endian header length, the
// dictionary padded with spaces and ended by '\n' to a multiple of 64
std::string NpzWriter::npy_header(const std::string& descr, const std::vector<int64_t>& shape) {
  std::string dict = "{'descr': '" + descr + "', 'fortran_order': False, 'shape': " + shape_string(shape) + ", }";
  const size_t unpadded = 10 + dict.size() + 1;
  dict.append((64 - unpadded % 64) % 64, ' ');
  dict.push_back('\n');
  std::string hdr = "\x93NUMPY";
  hdr.push_back('\x01');
  hdr.push_back('\x00');
  hdr.push_back((char)(dict.size() & 0xFF));
  hdr.push_back((char)((dict.size() >> 8) & 0xFF));
  return hdr + dict;
}

uint32_t NpzWriter::member_crc(const std::string& descr, const std::vector<int64_t>& shape, const void* data,
                               size_t bytes) {
  const std::string hdr = npy_header(descr, shape);
  return crc32_update(crc32_update(0, hdr.data(), hdr.size()), data, bytes);
}

bool NpzWriter::add_array(const std::string& name, const std::string& descr, const std::vector<int64_t>& shape,
                          const void* data, size_t bytes, const uint32_t* crc) {
  if (!err_.empty()) return false;
  const std::string hdr = npy_header(descr, shape);
  if (hdr.size() - 10 > 0xFFFF) return fail("npy header too long for " + name);

  Entry e;
  e.name = name + ".npy";
  e.size = hdr.size() + bytes;
  e.offset = pos_;
  e.zip64 = force_zip64_ || e.size >= k32Max;
  e.crc = crc ? *crc : crc32_update(crc32_update(0, hdr.data(), hdr.size()), data, bytes);

  unsigned char lh[30];
  auto w16 = [](unsigned char* p, uint32_t v) {
    p[0] = (unsigned char)(v & 0xFF);
    p[1] = (unsigned char)((v >> 8) & 0xFF);
  };
  auto w32 = [](unsigned char* p, uint32_t v) {
    for (int i = 0; i < 4; ++i) p[i] = (unsigned char)((v >> (8 * i)) & 0xFF);
  };
  w32(lh + 0, 0x04034b50u);
  w16(lh + 4, e.zip64 ? 45 : 20);  // version needed
  w16(lh + 6, 0);                  // flags
  w16(lh + 8, 0);                  // stored
  w16(lh + 10, dos_time_);
  w16(lh + 12, dos_date_);
  w32(lh + 14, e.crc);
  w32(lh + 18, e.zip64 ? (uint32_t)k32Max : (uint32_t)e.size);
  w32(lh + 22, e.zip64 ? (uint32_t)k32Max : (uint32_t)e.size);
  w16(lh + 26, (uint32_t)e.name.size());
  w16(lh + 28, e.zip64 ? 20 : 0);
  if (!put(lh, sizeof(lh)) || !put(e.name.data(), e.name.size())) return false;
  if (e.zip64) {
    unsigned char ex[20];
    w16(ex + 0, 0x0001);
    w16(ex + 2, 16);
    for (int i = 0; i < 8; ++i) ex[4 + i] = ex[12 + i] = (unsigned char)((e.size >> (8 * i)) & 0xFF);
    if (!put(ex, sizeof(ex))) return false;
  }
  if (!put(hdr.data(), hdr.size()) || !put(data, bytes)) return false;
  entries_.push_back(e);
  return true;
}

bool NpzWriter::add_f64(const std::string& name, double v) { return add_array(name, "<f8", {}, &v, sizeof(v)); }
bool NpzWriter::add_i64(const std::string& name, int64_t v) { return add_array(name, "<i8", {}, &v, sizeof(v)); }
bool NpzWriter::add_bool(const std::string& name, bool v) {
  const unsigned char b = v ? 1 : 0;
  return add_array(name, "|b1", {}, &b, 1);
}
bool NpzWriter::add_string(const std::string& name, const std::string& s) {
  const size_t len = s.empty() ? 1 : s.size();
  std::vector<uint32_t> u(len, 0u);
  for (size_t i = 0; i < s.size(); ++i) u[i] = (unsigned char)s[i];
  return add_array(name, "<U" + std::to_string(len), {}, u.data(), u.size() * sizeof(uint32_t));
}
bool NpzWriter::add_vector(const std::string& name, const double* v, int64_t n, const uint32_t* crc) {
  return add_array(name, "<f8", {n}, v, (size_t)n * sizeof(double), crc);
}

bool NpzWriter::close() {
  if (!f_) return fail("archive is not open");
  bool ok = err_.empty();
  const uint64_t cd_start = pos_;
  auto p16 = [&](uint32_t v) {
    unsigned char b[2] = {(unsigned char)(v & 0xFF), (unsigned char)((v >> 8) & 0xFF)};
    return put(b, 2);
  };
  auto p32 = [&](uint32_t v) {
    unsigned char b[4];
    for (int i = 0; i < 4; ++i) b[i] = (unsigned char)((v >> (8 * i)) & 0xFF);
    return put(b, 4);
  };
  auto p64 = [&](uint64_t v) {
    unsigned char b[8];
    for (int i = 0; i < 8; ++i) b[i] = (unsigned char)((v >> (8 * i)) & 0xFF);
    return put(b, 8);
  };
  for (const Entry& e : entries_) {
    if (!ok) break;
    const bool big_off = force_zip64_ || e.offset >= k32Max;
    const uint32_t extra = (e.zip64 || big_off) ? 4u + (e.zip64 ? 16u : 0u) + (big_off ? 8u : 0u) : 0u;
    const uint32_t ver = (e.zip64 || big_off) ? 45 : 20;
    ok = p32(0x02014b50u) && p16(ver) && p16(ver) && p16(0) && p16(0) && p16(dos_time_) && p16(dos_date_) &&
         p32(e.crc) && p32(e.zip64 ? (uint32_t)k32Max : (uint32_t)e.size) &&
         p32(e.zip64 ? (uint32_t)k32Max : (uint32_t)e.size) && p16((uint32_t)e.name.size()) && p16(extra) &&
         p16(0) && p16(0) && p16(0) && p32(0) && p32(big_off ? (uint32_t)k32Max : (uint32_t)e.offset) &&
         put(e.name.data(), e.name.size());
    if (ok && extra) {
      ok = p16(0x0001) && p16(extra - 4);
      if (ok && e.zip64) ok = p64(e.size) && p64(e.size);
      if (ok && big_off) ok = p64(e.offset);
    }
  }
  const uint64_t cd_size = pos_ - cd_start;
  const uint64_t count = entries_.size();
  const bool z64 = force_zip64_ || count >= 0xFFFF || cd_start >= k32Max || cd_size >= k32Max;
  if (ok && z64) {
    const uint64_t rec = pos_;
    ok = p32(0x06064b50u) && p64(44) && p16(45) && p16(45) && p32(0) && p32(0) && p64(count) && p64(count) &&
         p64(cd_size) && p64(cd_start) && p32(0x07064b50u) && p32(0) && p64(rec) && p32(1);
  }
  if (ok) {
    const uint32_t cnt16 = z64 ? 0xFFFFu : (uint32_t)count;
    ok = p32(0x06054b50u) && p16(0) && p16(0) && p16(cnt16) && p16(cnt16) &&
         p32(z64 ? (uint32_t)k32Max : (uint32_t)cd_size) && p32(z64 ? (uint32_t)k32Max : (uint32_t)cd_start) &&
         p16(0);
  }
  if (std::fclose(f_) != 0 && ok) ok = fail("close failed");
  f_ = nullptr;
  return ok && err_.empty();
}

}  // namespace hpr
