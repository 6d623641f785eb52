// npz.h -- reader for the tensormd potential file (.npz, stored or deflated).
//
// Replaces cnpy::npz_load (src/ML-TENSORMD/cnpy.cpp:191-272) for the keys the
// force path reads.  Unlike cnpy, values are converted by their stored dtype
// (cnpy's data<T>() reinterprets bytes, cnpy.h:41-45), so an int64 "nelt" or
// a float32 weight array is read correctly.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace tmd {

struct NpyArray {
  std::vector<size_t> shape;
  char kind = 'f';   // 'f' float, 'i' signed int, 'u' unsigned, 'b' bool
  int itemsize = 8;
  std::vector<double> d;  // every value as double (ints are exact up to 2^53)
  size_t size() const { return d.size(); }
  double scalar() const { return d.empty() ? 0.0 : d[0]; }
  int iscalar() const { return d.empty() ? 0 : static_cast<int>(d[0]); }
};

using Npz = std::map<std::string, NpyArray>;

// Throws std::runtime_error with a message on failure.
Npz load_npz(const std::string &path);

}  // namespace tmd
