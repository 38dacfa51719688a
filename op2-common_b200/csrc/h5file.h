// A self-contained reader and writer for the subset of the HDF5 file format
// that OP2's mesh files use (the HDF5 File Format Specification, version 2 and
// 3 documents of The HDF Group; no HDF5 library is linked).  Internal to
// libop2b; the OP2 entry points built on it are in op2b_hdf5.cpp.
//
// Reading: superblock versions 0-3 (a user block before it allowed), object
// headers version 1 and 2 with continuation blocks, groups as symbol tables
// (v1 B-trees, SNOD nodes, local heaps) or as link messages, datasets with
// compact, contiguous or chunked (v1 B-tree index) storage, chunk filters
// deflate, shuffle and fletcher32, fixed-point, floating-point and
// fixed-length string types of either byte order, attribute messages version
// 1-3.  Dense link or attribute storage (fractal heaps), other chunk indexes,
// variable-length and compound types are refused with an error.
//
// Writing: the layout HDF5 libraries write by default for these objects --
// superblock version 0, version-1 object headers, symbol-table groups,
// contiguous little-endian datasets with a version-3 layout message, version-1
// attribute messages.  A file is always written whole: changing an existing
// file reads its structure, applies the change and writes a new file (the raw
// data of unchanged datasets copied across), then renames it over the old one.
#pragma once

#include <cstdint>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace op2b {
namespace h5 {

struct Error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

enum class Cls : uint8_t { Fixed = 0, Float = 1, String = 3 };

struct Type {
  Cls cls = Cls::Fixed;
  uint32_t size = 0;        // bytes per element
  bool is_signed = true;    // fixed point
  bool big_endian = false;
  uint8_t str_pad = 0;      // string: 0 null-terminated, 1 null-padded, 2 space-padded
  static Type fixed(uint32_t bytes, bool sign = true);
  static Type real(uint32_t bytes);
  static Type str(uint32_t bytes);
  // "int", "long", "long long", "float", "double", "UNRECOGNISED" -- the names
  // OP2 gives the native types (op_hdf5_common.cpp:77-103)
  std::string op2_name() const;
};

struct Attr {
  std::string name;
  Type type;
  std::vector<uint64_t> dims;  // empty: scalar
  std::vector<uint8_t> data;   // elements in the type's byte order
  uint64_t count() const;
  // a string attribute's value without its padding
  std::string as_string() const;
};

struct Object {
  std::string name;  // the link name in the parent group
  bool group = false;
  std::vector<std::unique_ptr<Object>> children;  // groups
  std::vector<Attr> attrs;
  // datasets
  Type type;
  std::vector<uint64_t> dims;  // empty: scalar
  uint64_t count() const;      // elements
  uint64_t bytes() const { return count() * type.size; }
  // where the raw data is: in `mem` (written or compact), in a contiguous
  // extent of the source file, in chunks, or nowhere yet (fill value)
  enum class Store { Mem, Contiguous, Chunked, Unallocated } store = Store::Mem;
  std::vector<uint8_t> mem;
  uint64_t addr = 0;                 // contiguous data, or the chunk B-tree
  std::vector<uint32_t> chunk;       // chunk dims (rank + 1: last is the element size)
  struct Filter {
    uint16_t id;
    std::vector<uint32_t> cd;
  };
  std::vector<Filter> filters;
  std::vector<uint8_t> fill;         // fill value if defined (type.size bytes)

  Object *child(const std::string &n) const;
  const Attr *attr(const std::string &n) const;
  void set_attr(Attr a);  // replaces one of the same name
};

class File {
 public:
  // the structure of an existing file (raw data stays on disk until read)
  static std::unique_ptr<File> open(const std::string &path);
  static std::unique_ptr<File> create();
  ~File();

  Object &root() { return *root_; }
  // "/a/b/c" or "a/b/c"; nullptr when any component is missing
  Object *find(const std::string &path) const;
  // a new dataset at `path`, replacing one there, making the groups on the way
  // (OP2's create_path, op_hdf5_common.cpp:148-196); data holds count() *
  // type.size bytes in the type's byte order
  Object &put(const std::string &path, const Type &t, const std::vector<uint64_t> &dims,
              const void *data);

  // a dataset's elements in the file's type and byte order
  std::vector<uint8_t> read_raw(const Object &ds) const;
  // ... converted to `to` (numbers between fixed and floating point of any
  // size and byte order, as the library's conversion for native types does)
  std::vector<uint8_t> read(const Object &ds, const Type &to) const;

  // write the whole file to `path` (through a temporary file renamed over it)
  void save(const std::string &path) const;

 private:
  File() = default;
  struct Reader;
  std::unique_ptr<Object> root_;
  FILE *fp_ = nullptr;
  uint64_t base_ = 0;
  uint64_t fsize_ = 0;  // bytes in the source file: no structure may claim more
  int sa_ = 8, sl_ = 8;  // sizes of offsets and lengths in the source file
  friend struct Reader;
};

// convert `n` elements between two number types
void convert(const Type &from, const void *src, const Type &to, void *dst, uint64_t n);

}  // namespace h5
}  // namespace op2b
