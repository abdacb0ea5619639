// Reader and writer of the reference's graph binaries (csr_dag.bin and kin).
//
// The reference saves GraphCSR / GraphCOO with cereal's BinaryOutputArchive
// (include/Graph.h:132-148, 269-285, 300-316; cereal is fetched, not vendored,
// thirdparty/CMakeLists.txt:12-20).  This file restates that on-disk layout
// from cereal's published binary-archive rules, little-endian:
//   - arithmetic values and enums are written raw (enums as their 4-byte
//     underlying type);
//   - a std::vector<T> of arithmetic T is a uint64 element count, then the
//     elements' bytes;
//   - a std::shared_ptr<T> is a uint32 pointer id: 0 for null; the first
//     occurrence of a pointer carries id (k | 0x80000000), k = 1, 2, ... in
//     order of appearance, followed by the object; a repeated pointer carries
//     its k alone.
// The reference's records are then
//   CSR: uint32 version (1), uint32 format (0), int32 m, int64 nnz,
//        shared_ptr<vector<int64>> ptr, shared_ptr<vector<int32>> idx,
//        shared_ptr<vector<int32>> deg
//   COO: uint32 version (1), uint32 format (1), int32 m, int64 nnz,
//        shared_ptr<vector<int32>> row, shared_ptr<vector<int32>> col
// No file written by the reference ships with it, so the layout is checked
// against fixtures built from these rules, not against reference output.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.cuh"

namespace gary {
namespace {

constexpr uint32_t kCerealNew = 0x80000000u;
constexpr uint32_t kSerDesV1 = 1;
constexpr uint32_t kFormatCSR = 0, kFormatCOO = 1;

struct File {
  FILE *f = nullptr;
  explicit File(const char *path, const char *mode) : f(std::fopen(path, mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

// Reads exactly `bytes` or reports the truncation.
int get(FILE *f, void *dst, size_t bytes, const char *what) {
  if (bytes && std::fread(dst, 1, bytes, f) != bytes) {
    set_error("graph binary truncated while reading %s", what);
    return GARY_ERR_INPUT;
  }
  return GARY_OK;
}

struct Header {
  uint32_t version, format;
  int32_t m;
  int64_t nnz;
};

int read_header(FILE *f, Header &h) {
  GARY_TRY(get(f, &h.version, 4, "the version"));
  GARY_TRY(get(f, &h.format, 4, "the format tag"));
  GARY_TRY(get(f, &h.m, 4, "the vertex count"));
  GARY_TRY(get(f, &h.nnz, 8, "the edge count"));
  if (h.version != kSerDesV1) {
    set_error("graph binary version %u is not supported (expected 1)", h.version);
    return GARY_ERR_INPUT;
  }
  if (h.format != kFormatCSR && h.format != kFormatCOO) {
    set_error("graph binary format tag %u is neither CSR (0) nor COO (1)", h.format);
    return GARY_ERR_INPUT;
  }
  if (h.m < 0 || h.nnz < 0) {
    set_error("graph binary has negative sizes (m %d, nnz %lld)", h.m, (long long)h.nnz);
    return GARY_ERR_INPUT;
  }
  return GARY_OK;
}

// One shared_ptr<vector<T>> field, the k-th pointer of the archive.  With
// dst == nullptr the elements are skipped; `count` receives the length.
template <typename T>
int read_vector_ptr(FILE *f, uint32_t k, const char *what, T *dst, uint64_t cap, uint64_t &count) {
  uint32_t id = 0;
  GARY_TRY(get(f, &id, 4, what));
  if (id != (k | kCerealNew)) {
    set_error("graph binary: %s has pointer id 0x%08x (expected a new pointer 0x%08x)", what, id,
              k | kCerealNew);
    return GARY_ERR_INPUT;
  }
  GARY_TRY(get(f, &count, 8, what));
  if (!dst) {  // skipped, but read through, so a truncated file is noticed
    T buf[4096];
    for (uint64_t left = count; left;) {
      const uint64_t k = left < 4096 ? left : 4096;
      GARY_TRY(get(f, buf, k * sizeof(T), what));
      left -= k;
    }
    return GARY_OK;
  }
  if (count > cap) {
    set_error("graph binary: %s holds %llu entries, buffer holds %llu", what,
              (unsigned long long)count, (unsigned long long)cap);
    return GARY_ERR_INVALID;
  }
  return get(f, dst, count * sizeof(T), what);
}

template <typename T>
int write_vector_ptr(FILE *f, uint32_t k, const T *src, uint64_t count) {
  const uint32_t id = k | kCerealNew;
  if (std::fwrite(&id, 4, 1, f) != 1 || std::fwrite(&count, 8, 1, f) != 1 ||
      (count && std::fwrite(src, sizeof(T), count, f) != count)) {
    set_error("writing the graph binary failed");
    return GARY_ERR_INPUT;
  }
  return GARY_OK;
}

}  // namespace
}  // namespace gary

using gary::Header;

extern "C" int gary_bin_info(const char *path, uint32_t *format, uint32_t *n, uint64_t *nnz) {
  GARY_CHECK_ARG(path && format && n && nnz, "NULL argument");
  gary::clear_error();
  gary::File f(path, "rb");
  if (!f.f) {
    gary::set_error("cannot open graph binary '%s'", path);
    return GARY_ERR_INPUT;
  }
  Header h;
  GARY_TRY(gary::read_header(f.f, h));
  *format = h.format;
  *n = (uint32_t)h.m;
  *nnz = (uint64_t)h.nnz;
  return GARY_OK;
}

extern "C" int gary_bin_read_csr(const char *path, uint64_t *ptr, uint32_t *idx) {
  GARY_CHECK_ARG(path && ptr, "NULL argument");
  gary::clear_error();
  gary::File f(path, "rb");
  if (!f.f) {
    gary::set_error("cannot open graph binary '%s'", path);
    return GARY_ERR_INPUT;
  }
  Header h;
  GARY_TRY(gary::read_header(f.f, h));
  GARY_CHECK_ARG(h.format == gary::kFormatCSR, "graph binary holds a COO graph, not a CSR");
  GARY_CHECK_ARG(h.nnz == 0 || idx, "idx is NULL");
  uint64_t np = 0, ni = 0, nd = 0;
  GARY_TRY(gary::read_vector_ptr<uint64_t>(f.f, 1, "ptr", ptr, (uint64_t)h.m + 1, np));
  GARY_TRY(gary::read_vector_ptr<uint32_t>(f.f, 2, "idx", idx, (uint64_t)h.nnz, ni));
  GARY_TRY(gary::read_vector_ptr<uint32_t>(f.f, 3, "deg", (uint32_t *)nullptr, 0, nd));
  if (np != (uint64_t)h.m + 1 || ni != (uint64_t)h.nnz || (nd != (uint64_t)h.m && nd != 0) ||
      ptr[0] != 0 || ptr[h.m] != (uint64_t)h.nnz) {
    gary::set_error("graph binary CSR is inconsistent (m %d, nnz %lld, |ptr| %llu, |idx| %llu, |deg| %llu)",
                    h.m, (long long)h.nnz, (unsigned long long)np, (unsigned long long)ni,
                    (unsigned long long)nd);
    return GARY_ERR_INPUT;
  }
  return GARY_OK;
}

extern "C" int gary_bin_read_coo(const char *path, uint32_t *src, uint32_t *dst) {
  GARY_CHECK_ARG(path, "NULL argument");
  gary::clear_error();
  gary::File f(path, "rb");
  if (!f.f) {
    gary::set_error("cannot open graph binary '%s'", path);
    return GARY_ERR_INPUT;
  }
  Header h;
  GARY_TRY(gary::read_header(f.f, h));
  GARY_CHECK_ARG(h.format == gary::kFormatCOO, "graph binary holds a CSR graph, not a COO");
  GARY_CHECK_ARG(h.nnz == 0 || (src && dst), "src/dst is NULL");
  uint64_t nr = 0, nc = 0;
  GARY_TRY(gary::read_vector_ptr<uint32_t>(f.f, 1, "row", src, (uint64_t)h.nnz, nr));
  GARY_TRY(gary::read_vector_ptr<uint32_t>(f.f, 2, "col", dst, (uint64_t)h.nnz, nc));
  if (nr != (uint64_t)h.nnz || nc != (uint64_t)h.nnz) {
    gary::set_error("graph binary COO is inconsistent (nnz %lld, |row| %llu, |col| %llu)",
                    (long long)h.nnz, (unsigned long long)nr, (unsigned long long)nc);
    return GARY_ERR_INPUT;
  }
  return GARY_OK;
}

extern "C" int gary_bin_write_csr(const char *path, const uint64_t *ptr, const uint32_t *idx, uint32_t n,
                                  uint64_t nnz) {
  GARY_CHECK_ARG(path && ptr && (nnz == 0 || idx), "NULL argument");
  GARY_CHECK_ARG(n < 0x80000000u && nnz < 0x8000000000000000ull, "sizes exceed the format's signed fields");
  GARY_CHECK_ARG(ptr[0] == 0 && ptr[n] == nnz, "ptr[0] must be 0 and ptr[n] must equal nnz");
  gary::clear_error();
  gary::File f(path, "wb");
  if (!f.f) {
    gary::set_error("cannot create graph binary '%s'", path);
    return GARY_ERR_INPUT;
  }
  const uint32_t hv[2] = {gary::kSerDesV1, gary::kFormatCSR};
  const int32_t m = (int32_t)n;
  const int64_t z = (int64_t)nnz;
  if (std::fwrite(hv, 4, 2, f.f) != 2 || std::fwrite(&m, 4, 1, f.f) != 1 || std::fwrite(&z, 8, 1, f.f) != 1) {
    gary::set_error("writing the graph binary failed");
    return GARY_ERR_INPUT;
  }
  std::vector<uint32_t> deg(n);
  for (uint32_t v = 0; v < n; ++v) deg[v] = (uint32_t)(ptr[v + 1] - ptr[v]);
  GARY_TRY(gary::write_vector_ptr(f.f, 1, ptr, (uint64_t)n + 1));
  GARY_TRY(gary::write_vector_ptr(f.f, 2, idx, nnz));
  GARY_TRY(gary::write_vector_ptr(f.f, 3, deg.data(), (uint64_t)n));
  return GARY_OK;
}
