// serialize_dump -- writes and reads the on-disk form of the C++ drop-in
// container CRSMatrix<RangeDynamic, bool, uint32_t, TSize> (its header alone,
// no library), for the byte-format test.
//
//   serialize_dump write <u64|u32> ncols nnz entries.bin rowmap.bin out.bin
//       builds the matrix from raw little-endian arrays (entries uint32,
//       rowmap uint64) and writes matrix.serialize(out)
//   serialize_dump reload <u64|u32> in.bin out.bin
//       matrix.load(in), then matrix.serialize(out)
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <vector>

#include "diverg/crs_matrix.hpp"

template <typename T>
static std::vector<T> read_raw(const char* path) {
  std::ifstream f(path, std::ios::binary);
  std::vector<char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  std::vector<T> v(b.size() / sizeof(T));
  std::memcpy(v.data(), b.data(), v.size() * sizeof(T));
  return v;
}

template <typename TSize>
static int run(int argc, char** argv) {
  using M = diverg::CRSMatrix<diverg::crs_matrix::RangeDynamic, bool, uint32_t, TSize>;
  const std::string mode = argv[1];
  if (mode == "write" && argc == 8) {
    const uint32_t ncols = uint32_t(std::strtoull(argv[3], nullptr, 10));
    const uint64_t nnz = std::strtoull(argv[4], nullptr, 10);
    std::vector<uint32_t> e = read_raw<uint32_t>(argv[5]);
    std::vector<uint64_t> r64 = read_raw<uint64_t>(argv[6]);
    std::vector<TSize> r(r64.begin(), r64.end());
    M m(ncols, std::move(e), std::move(r), TSize(nnz));
    std::ofstream out(argv[7], std::ios::binary);
    m.serialize(out);
    return out.good() ? 0 : 2;
  }
  if (mode == "reload" && argc == 5) {
    M m;
    std::ifstream in(argv[3], std::ios::binary);
    m.load(in);
    if (!in.good()) return 3;
    std::ofstream out(argv[4], std::ios::binary);
    m.serialize(out);
    return out.good() ? 0 : 2;
  }
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 3) return 1;
  if (!std::strcmp(argv[2], "u64")) return run<uint64_t>(argc, argv);
  if (!std::strcmp(argv[2], "u32")) return run<uint32_t>(argc, argv);
  return 1;
}
