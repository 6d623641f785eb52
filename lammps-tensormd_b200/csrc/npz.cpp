// npz.cpp -- zip (central directory, zip64 extras) + NPY v1/v2/v3 parsing.
#include "npz.h"

#include <zlib.h>

#include <cstring>
#include <fstream>
#include <stdexcept>

namespace tmd {

namespace {

uint16_t rd16(const unsigned char *p) { return uint16_t(p[0] | (p[1] << 8)); }
uint32_t rd32(const unsigned char *p) {
  return uint32_t(p[0]) | (uint32_t(p[1]) << 8) | (uint32_t(p[2]) << 16) |
         (uint32_t(p[3]) << 24);
}
uint64_t rd64(const unsigned char *p) {
  return uint64_t(rd32(p)) | (uint64_t(rd32(p + 4)) << 32);
}

[[noreturn]] void fail(const std::string &m) { throw std::runtime_error(m); }

std::vector<unsigned char> inflate_raw(const unsigned char *src, size_t n,
                                       size_t out_n) {
  std::vector<unsigned char> out(out_n);
  z_stream zs;
  std::memset(&zs, 0, sizeof(zs));
  if (inflateInit2(&zs, -MAX_WBITS) != Z_OK) fail("npz: inflateInit2 failed");
  zs.next_in = const_cast<unsigned char *>(src);
  zs.avail_in = static_cast<uInt>(n);
  zs.next_out = out.data();
  zs.avail_out = static_cast<uInt>(out_n);
  int rc = inflate(&zs, Z_FINISH);
  inflateEnd(&zs);
  if (rc != Z_STREAM_END) fail("npz: deflate stream is corrupt");
  return out;
}

NpyArray parse_npy(const unsigned char *p, size_t n, const std::string &key) {
  if (n < 10 || std::memcmp(p, "\x93NUMPY", 6) != 0)
    fail("npz: entry " + key + " is not an NPY array");
  int major = p[6];
  size_t hlen, hoff;
  if (major == 1) {
    hlen = rd16(p + 8);
    hoff = 10;
  } else {
    hlen = rd32(p + 8);
    hoff = 12;
  }
  if (hoff + hlen > n) fail("npz: truncated header in " + key);
  std::string h(reinterpret_cast<const char *>(p + hoff), hlen);
  NpyArray a;
  auto dpos = h.find("'descr'");
  if (dpos == std::string::npos) fail("npz: no descr in " + key);
  auto q1 = h.find('\'', h.find(':', dpos));
  auto q2 = h.find('\'', q1 + 1);
  std::string descr = h.substr(q1 + 1, q2 - q1 - 1);
  if (descr.size() < 3) fail("npz: bad descr in " + key);
  char endian = descr[0];
  a.kind = descr[1];
  a.itemsize = std::stoi(descr.substr(2));
  if (endian == '>') fail("npz: big-endian arrays are not supported (" + key + ")");
  bool fortran = h.find("'fortran_order': True") != std::string::npos;
  auto spos = h.find('(', h.find("'shape'"));
  auto send = h.find(')', spos);
  std::string sh = h.substr(spos + 1, send - spos - 1);
  size_t count = 1;
  size_t i = 0;
  while (i < sh.size()) {
    while (i < sh.size() && (sh[i] == ' ' || sh[i] == ',')) i++;
    if (i >= sh.size()) break;
    size_t j = i;
    while (j < sh.size() && sh[j] >= '0' && sh[j] <= '9') j++;
    if (j == i) break;
    size_t v = std::stoull(sh.substr(i, j - i));
    a.shape.push_back(v);
    count *= v;
    i = j;
  }
  if (fortran && a.shape.size() > 1) fail("npz: Fortran-ordered array " + key);
  const unsigned char *data = p + hoff + hlen;
  if (hoff + hlen + count * a.itemsize > n) fail("npz: truncated data in " + key);
  a.d.resize(count);
  for (size_t k = 0; k < count; k++) {
    const unsigned char *e = data + k * a.itemsize;
    double v = 0;
    if (a.kind == 'f') {
      if (a.itemsize == 8) { double t; std::memcpy(&t, e, 8); v = t; }
      else if (a.itemsize == 4) { float t; std::memcpy(&t, e, 4); v = t; }
      else fail("npz: unsupported float width in " + key);
    } else if (a.kind == 'i') {
      if (a.itemsize == 8) { int64_t t; std::memcpy(&t, e, 8); v = double(t); }
      else if (a.itemsize == 4) { int32_t t; std::memcpy(&t, e, 4); v = t; }
      else if (a.itemsize == 2) { int16_t t; std::memcpy(&t, e, 2); v = t; }
      else if (a.itemsize == 1) { int8_t t; std::memcpy(&t, e, 1); v = t; }
      else fail("npz: unsupported int width in " + key);
    } else if (a.kind == 'u' || a.kind == 'b') {
      uint64_t t = 0;
      std::memcpy(&t, e, a.itemsize <= 8 ? a.itemsize : 8);
      v = double(t);
    } else {
      fail("npz: unsupported dtype " + descr + " in " + key);
    }
    a.d[k] = v;
  }
  return a;
}

}  // namespace

Npz load_npz(const std::string &path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) fail("cannot open potential file " + path);
  std::vector<unsigned char> buf((std::istreambuf_iterator<char>(in)),
                                 std::istreambuf_iterator<char>());
  const size_t n = buf.size();
  if (n < 22) fail("npz: file too small: " + path);
  // end of central directory
  size_t eocd = std::string::npos;
  for (size_t i = n - 22 + 1; i-- > 0;) {
    if (rd32(&buf[i]) == 0x06054b50u) { eocd = i; break; }
    if (n - i > 65557) break;
  }
  if (eocd == std::string::npos) fail("npz: no end-of-central-directory in " + path);
  uint64_t nent = rd16(&buf[eocd + 10]);
  uint64_t cd_off = rd32(&buf[eocd + 16]);
  if (cd_off == 0xFFFFFFFFu || nent == 0xFFFF) {
    // zip64 end-of-central-directory locator precedes the EOCD
    if (eocd < 20 || rd32(&buf[eocd - 20]) != 0x07064b50u) fail("npz: bad zip64 locator");
    uint64_t z64 = rd64(&buf[eocd - 20 + 8]);
    if (z64 + 56 > n || rd32(&buf[z64]) != 0x06064b50u) fail("npz: bad zip64 record");
    nent = rd64(&buf[z64 + 32]);
    cd_off = rd64(&buf[z64 + 48]);
  }
  Npz out;
  size_t p = cd_off;
  for (uint64_t e = 0; e < nent; e++) {
    if (p + 46 > n || rd32(&buf[p]) != 0x02014b50u) fail("npz: bad central directory");
    uint16_t method = rd16(&buf[p + 10]);
    uint64_t csize = rd32(&buf[p + 20]);
    uint64_t usize = rd32(&buf[p + 24]);
    uint16_t nlen = rd16(&buf[p + 28]);
    uint16_t xlen = rd16(&buf[p + 30]);
    uint16_t clen = rd16(&buf[p + 32]);
    uint64_t loff = rd32(&buf[p + 42]);
    std::string name(reinterpret_cast<const char *>(&buf[p + 46]), nlen);
    // zip64 extra field
    size_t x = p + 46 + nlen, xe = x + xlen;
    while (x + 4 <= xe) {
      uint16_t id = rd16(&buf[x]), sz = rd16(&buf[x + 2]);
      if (id == 0x0001) {
        size_t q = x + 4;
        if (usize == 0xFFFFFFFFu) { usize = rd64(&buf[q]); q += 8; }
        if (csize == 0xFFFFFFFFu) { csize = rd64(&buf[q]); q += 8; }
        if (loff == 0xFFFFFFFFu) { loff = rd64(&buf[q]); q += 8; }
      }
      x += 4 + sz;
    }
    p = xe + clen;
    if (loff + 30 > n || rd32(&buf[loff]) != 0x04034b50u) fail("npz: bad local header");
    size_t doff = loff + 30 + rd16(&buf[loff + 26]) + rd16(&buf[loff + 28]);
    if (doff + csize > n) fail("npz: truncated entry " + name);
    std::string key = name;
    if (key.size() > 4 && key.compare(key.size() - 4, 4, ".npy") == 0)
      key = key.substr(0, key.size() - 4);
    if (method == 0) {
      out[key] = parse_npy(&buf[doff], csize, key);
    } else if (method == 8) {
      auto raw = inflate_raw(&buf[doff], csize, usize);
      out[key] = parse_npy(raw.data(), raw.size(), key);
    } else {
      fail("npz: unsupported compression method in " + name);
    }
  }
  return out;
}

}  // namespace tmd
