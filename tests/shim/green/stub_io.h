// Raw arrays written by tests/test_shim.py for the green-mbpt stand-ins: <name>.bin (little-endian
// doubles or int64) next to <name>.shape (the dimensions, whitespace separated).  Test infrastructure.
#pragma once
#include <complex>
#include <cstdint>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace green::stub {

inline std::vector<size_t> shape_of(const std::string& base) {
  std::ifstream f(base + ".shape");
  if (!f) throw std::runtime_error("missing " + base + ".shape");
  std::vector<size_t> s;
  size_t x;
  while (f >> x) s.push_back(x);
  return s;
}

template <typename T>
std::vector<T> load(const std::string& base) {
  std::ifstream f(base + ".bin", std::ios::binary | std::ios::ate);
  if (!f) throw std::runtime_error("missing " + base + ".bin");
  const size_t bytes = (size_t)f.tellg();
  std::vector<T> v(bytes / sizeof(T));
  f.seekg(0);
  f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)bytes);
  return v;
}

template <typename T>
void save(const std::string& base, const T* p, size_t n) {
  std::ofstream f(base + ".bin", std::ios::binary);
  f.write(reinterpret_cast<const char*>(p), (std::streamsize)(n * sizeof(T)));
}

}  // namespace green::stub
