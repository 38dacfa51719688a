// OP2's HDF5 mesh I/O: the entry points of op2/include/op_hdf5.h
// (op2/src/externlib/op_hdf5.cpp:66-1121, op_hdf5_common.cpp) over the
// file-format code of h5file.cpp, plus host-only op2b_h5_* helpers.
//
// A read declares what it found through op_decl_set / op_decl_map /
// op_decl_dat_char, which upload it.  A write fetches the device values
// first.  File layouts follow the reference: a set is a one-element int
// dataset named after the set; a map a [from size][dim] dataset with int
// attributes "size" (from size) and "dim" and a string attribute "type"; a
// dat a [set size][dim] dataset with "size" (bytes per element, as the
// reference stores dat->size), "dim" and "type"; a constant a [dim] dataset
// with "dim" and "type".  Where the reference exits the program on an error,
// these functions record it (op2b_last_error) and return without declaring
// or writing anything.
#include <sys/stat.h>

#include <cstdio>
#include <exception>
#include <cstring>
#include <string>
#include <vector>

#include "h5file.h"
#include "op2b_runtime.h"

using namespace op2b;
namespace H = op2b::h5;

namespace {

bool file_exists(const char *f) {
  struct stat st;
  return f && stat(f, &st) == 0;
}

// op_type_equivalence (op2/src/externlib/op_util.cpp:240-276): the names of
// double, float and int that OP2 treats as one type
int type_class(const std::string &t) {
  static const char *d[] = {"double", "double:soa", "real(8)", "double precision"};
  static const char *f[] = {"float", "float:soa", "real(4)", "real"};
  static const char *i[] = {"int", "int:soa", "integer(4)", "integer"};
  for (int k = 0; k < 4; k++) {
    if (t == d[k]) return 1;
    if (t == f[k]) return 2;
    if (t == i[k]) return 3;
  }
  return 0;
}
bool type_equivalent(const std::string &a, const std::string &b) {
  int ca = type_class(a);
  return ca != 0 && ca == type_class(b);
}

// the file type of an OP2 type name (op_hdf5.cpp's strcmp chains: "double",
// "double:soa", "double precision", "real(8)"; ... "long long:soa"); false
// for names it does not know
bool h5_type(const std::string &t, H::Type &out) {
  switch (type_class(t)) {
    case 1:
      out = H::Type::real(8);
      return true;
    case 2:
      out = H::Type::real(4);
      return true;
    case 3:
      out = H::Type::fixed(4);
      return true;
  }
  if (t == "long" || t == "long:soa" || t == "long long" || t == "long long:soa") {
    out = H::Type::fixed(8);
    return true;
  }
  return false;
}

// the name op_write_const_hdf5 stores for a type (op_hdf5.cpp:783-800)
std::string stored_name(const std::string &t) {
  switch (type_class(t)) {
    case 1:
      return "double";
    case 2:
      return "float";
    case 3:
      return "int";
  }
  return t;
}

H::Attr int_attr(const char *name, int v) {
  H::Attr a;
  a.name = name;
  a.type = H::Type::fixed(4);
  a.dims = {1};
  a.data.resize(4);
  memcpy(a.data.data(), &v, 4);
  return a;
}

// a fixed-length string attribute of `width` bytes (null-padded)
H::Attr str_attr(const char *name, const std::string &v, size_t width) {
  H::Attr a;
  a.name = name;
  a.type = H::Type::str((uint32_t)std::max<size_t>(width, 1));
  a.data.assign(a.type.size, 0);
  memcpy(a.data.data(), v.data(), std::min<size_t>(v.size(), a.type.size));
  return a;
}

bool int_attr_of(const H::Object &o, const char *name, long long &v) {
  const H::Attr *a = o.attr(name);
  if (!a || a->type.cls == H::Cls::String || a->count() < 1) return false;
  H::convert(a->type, a->data.data(), H::Type::fixed(8), &v, 1);
  return true;
}

// size (first dimension) and dim (second, 1 for a one-dimensional dataset)
// as get_dataset_properties reports them (op_hdf5_common.cpp:105-146)
void props(const H::Object &o, long long &size, long long &dim) {
  if (o.dims.empty()) {
    size = dim = 0;
    return;
  }
  size = (long long)o.dims[0];
  dim = o.dims.size() > 1 ? (long long)o.dims[1] : 1;
}

std::unique_ptr<H::File> open_or_fail(const char *file, const char *who) {
  if (!file_exists(file)) {
    set_error("%s: file %s does not exist", who, file ? file : "(null)");
    return nullptr;
  }
  return H::File::open(file);
}

// current device values of a dat in the current numbering
bool dat_values(op_dat d, std::vector<char> &buf) {
  buf.resize((size_t)d->set->size * d->size);
  if (buf.empty()) return true;
  return download_host(buf.data(), d->data_d, buf.size(), "op_dump_to_hdf5");
}

}  // namespace

extern "C" {

op_set op_decl_set_hdf5(char const *file, char const *name) {
  try {
    auto f = open_or_fail(file, "op_decl_set_hdf5");
    if (!f) return nullptr;
    H::Object *o = f->find(name ? name : "");
    if (!o || o->group || o->count() < 1) {
      set_error("op_decl_set_hdf5: no set size '%s' in file %s", name ? name : "", file);
      return nullptr;
    }
    std::vector<uint8_t> v = f->read(*o, H::Type::fixed(4));
    int size;
    memcpy(&size, v.data(), 4);
    return op_decl_set(size, name);
  } catch (const std::exception &e) {
    set_error("op_decl_set_hdf5: %s: %s", file, e.what());
    return nullptr;
  }
}

op_set op_decl_set_hdf5_infer_size(char const *file, char const *name,
                                   char const *set_dataset_name) {
  try {
    auto f = open_or_fail(file, "op_decl_set_hdf5_infer_size");
    if (!f) return nullptr;
    H::Object *o = f->find(set_dataset_name ? set_dataset_name : "");
    if (!o || o->group) {
      set_error("op_decl_set_hdf5_infer_size: dataset '%s' not found in file '%s'",
                set_dataset_name ? set_dataset_name : "", file);
      return nullptr;
    }
    long long size, dim;
    props(*o, size, dim);
    return op_decl_set((int)size, name);
  } catch (const std::exception &e) {
    set_error("op_decl_set_hdf5_infer_size: %s: %s", file, e.what());
    return nullptr;
  }
}

op_map op_decl_map_hdf5(op_set from, op_set to, int dim, char const *file, char const *name) {
  try {
    if (!from || !to) {
      set_error("op_decl_map_hdf5: invalid 'from'/'to' set for map %s", name ? name : "");
      return nullptr;
    }
    auto f = open_or_fail(file, "op_decl_map_hdf5");
    if (!f) return nullptr;
    H::Object *o = f->find(name ? name : "");
    if (!o || o->group) {
      set_error("op_map with name : %s not found in file : %s", name ? name : "", file);
      return nullptr;
    }
    long long size, mdim;
    props(*o, size, mdim);
    if (size != from->size) {
      set_error("map from set size %lld in file %s and size %d do not match", size, file,
                from->size);
      return nullptr;
    }
    if (mdim != dim) {
      set_error("map.dim %lld in file %s and dim %d do not match", mdim, file, dim);
      return nullptr;
    }
    std::string typ = o->type.op2_name();
    if (typ != "int" && typ != "long") {
      set_error("Unknown type in file %s for map %s", file, name);
      return nullptr;
    }
    // 64-bit maps are read as 64-bit and narrowed: libop2b's maps are int
    std::vector<uint8_t> v = f->read(*o, H::Type::fixed(8));
    std::vector<int> m((size_t)size * dim);
    const long long *w = (const long long *)v.data();
    for (size_t i = 0; i < m.size(); i++) {
      if (w[i] < INT32_MIN || w[i] > INT32_MAX) {
        set_error("op_decl_map_hdf5: map %s in file %s holds %lld, outside int", name, file,
                  w[i]);
        return nullptr;
      }
      m[i] = (int)w[i];
    }
    return op_decl_map(from, to, dim, m.empty() ? nullptr : m.data(), name);
  } catch (const std::exception &e) {
    set_error("op_decl_map_hdf5: %s: %s", file, e.what());
    return nullptr;
  }
}

op_dat op_decl_dat_hdf5(op_set set, int dim, char const *type, char const *file,
                        char const *name) {
  try {
    if (!set || !type) {
      set_error("op_decl_dat_hdf5: invalid set or type for data %s", name ? name : "");
      return nullptr;
    }
    auto f = open_or_fail(file, "op_decl_dat_hdf5");
    if (!f) return nullptr;
    H::Object *o = f->find(name ? name : "");
    if (!o || o->group) {
      set_error("op_dat with name : %s not found in file : %s", name ? name : "", file);
      return nullptr;
    }
    long long size, ddim;
    props(*o, size, ddim);
    if (ddim != dim) {
      set_error("dat.dim %lld in file %s and dim %d do not match", ddim, file, dim);
      return nullptr;
    }
    if (size != set->size) {
      set_error("op_decl_dat_hdf5: dat %s has %lld elements in file %s, its set %d", name, size,
                file, set->size);
      return nullptr;
    }
    H::Type want;
    if (!h5_type(type, want)) {
      set_error("unknown type for dat");
      return nullptr;
    }
    std::string typ = o->type.op2_name();
    if (!type_equivalent(typ, type) && rt().opt_diags > 0)
      printf("dat.type %s in file %s and type %s do not match, performing automatic "
             "conversion\n", typ.c_str(), file, type);
    std::vector<uint8_t> v = f->read(*o, want);
    return op_decl_dat_char(set, dim, type, (int)want.size, v.empty() ? nullptr : (char *)v.data(),
                            name);
  } catch (const std::exception &e) {
    set_error("op_decl_dat_hdf5: %s: %s", file, e.what());
    return nullptr;
  }
}

void op_get_const_hdf5(char const *name, int dim, char const *type, char *const_data,
                       char const *file_name) {
  try {
    auto f = open_or_fail(file_name, "op_get_const_hdf5");
    if (!f) return;
    H::Object *o = f->find(name ? name : "");
    if (!o || o->group) {
      set_error("dataset '%s' not found in file '%s'", name ? name : "", file_name);
      return;
    }
    long long cdim = 0;
    if (!int_attr_of(*o, "dim", cdim) || cdim != dim) {
      set_error("dim of constant %lld in file %s and requested dim %d do not match", cdim,
                file_name, dim);
      return;
    }
    const H::Attr *ta = o->attr("type");
    std::string typ = ta && ta->type.cls == H::Cls::String ? ta->as_string() : "";
    if (!type_equivalent(typ, type)) {
      if (rt().opt_diags > 0)
        printf("type of constant %s in file %s and requested type %s do not match, performing "
               "automatic type conversion\n", typ.c_str(), file_name, type);
      typ = type;
    }
    H::Type want;
    if (!h5_type(typ, want)) {
      set_error("Unknown type in file %s for constant %s", file_name, name);
      return;
    }
    if (o->count() < (uint64_t)dim) {
      set_error("op_get_const_hdf5: constant %s in file %s has %llu values, not %d", name,
                file_name, (unsigned long long)o->count(), dim);
      return;
    }
    std::vector<uint8_t> v = f->read(*o, want);
    memcpy(const_data, v.data(), (size_t)dim * want.size);
  } catch (const std::exception &e) {
    set_error("op_get_const_hdf5: %s: %s", file_name, e.what());
  }
}

void op_dump_to_hdf5(char const *file_name) {
  Runtime &r = rt();
  if (!r.ready()) return;
  if (r.opt_diags > 0) printf("Writing to %s\n", file_name);
  try {
    auto f = H::File::create();
    for (auto &s : r.sets) {
      int size = s->size;
      f->put(s->name, H::Type::fixed(4), {1}, &size);
    }
    for (auto &m : r.maps) {
      std::vector<int> h((size_t)m->from->size * m->dim);
      if (!h.empty() &&
          !download_host(h.data(), m->map_d, h.size() * sizeof(int), "op_dump_to_hdf5"))
        return;
      H::Object &o = f->put(m->name, H::Type::fixed(4),
                            {(uint64_t)m->from->size, (uint64_t)m->dim}, h.data());
      o.set_attr(int_attr("size", m->from->size));
      o.set_attr(int_attr("dim", m->dim));
      o.set_attr(str_attr("type", "int", 10));
    }
    for (auto &d : r.dats) {
      H::Type t;
      if (!h5_type(d->type, t) || (int)t.size * d->dim != d->size) {
        set_error("Unknown type for data elements %s", d->type);
        return;
      }
      std::vector<char> buf;
      if (!dat_values(d.get(), buf)) return;
      H::Object &o = f->put(d->name, t, {(uint64_t)d->set->size, (uint64_t)d->dim}, buf.data());
      o.set_attr(int_attr("size", d->size));
      o.set_attr(int_attr("dim", d->dim));
      o.set_attr(str_attr("type", d->type, strlen(d->type)));
    }
    f->save(file_name);
  } catch (const std::exception &e) {
    set_error("op_dump_to_hdf5: %s: %s", file_name, e.what());
  }
}

void op_write_const_hdf5(char const *name, int dim, char const *type, char *const_data,
                         char const *file_name) {
  if (rt().opt_diags > 0) printf("Writing '%s' to file '%s'\n", name, file_name);
  try {
    H::Type t;
    if (!type || !h5_type(type, t)) {
      set_error("Unknown type %s for constant %s: cannot write constant to file",
                type ? type : "(null)", name ? name : "");
      return;
    }
    auto f = file_exists(file_name) ? H::File::open(file_name) : H::File::create();
    if (f->find(name ? name : "")) {
      set_error("op_write_const_hdf5: %s already holds '%s'", file_name, name);
      return;
    }
    H::Object &o = f->put(name ? name : "", t, {(uint64_t)dim}, const_data);
    o.set_attr(int_attr("dim", dim));
    o.set_attr(str_attr("type", stored_name(type), strlen(type)));
    f->save(file_name);
  } catch (const std::exception &e) {
    set_error("op_write_const_hdf5: %s: %s", file_name, e.what());
  }
}

// op_fetch_data_hdf5 (op_hdf5.cpp:882-1085): the dat's values in the order the
// application declared them, written into the dataset at `path_name` -- an
// existing one after checking its size, dim and type attributes, else a new
// one (with the groups on its path) -- in a file created if missing
void op_fetch_data_hdf5_file_path(op_dat dat, char const *file_name, char const *path_name) {
  Runtime &r = rt();
  if (!r.ready()) return;
  if (!dat || !path_name) {
    set_error("op_fetch_data_hdf5_file: invalid dat or path");
    return;
  }
  if (r.opt_diags > 0) printf("Writing '%s' to file '%s'\n", path_name, file_name);
  try {
    H::Type t;
    if (!h5_type(dat->type, t) || (int)t.size * dat->dim != dat->size) {
      set_error("Unknown type for data elements");
      return;
    }
    std::vector<char> buf((size_t)dat->set->size * dat->size);
    if (!buf.empty()) fetch_original_order(dat, buf.data(), 0, dat->set->size - 1);
    auto f = file_exists(file_name) ? H::File::open(file_name) : H::File::create();
    std::vector<uint64_t> dims = {(uint64_t)dat->set->size, (uint64_t)dat->dim};
    H::Object *o = f->find(path_name);
    if (o && !o->group) {
      long long v;
      if (!int_attr_of(*o, "size", v)) {
        set_error("data set %s on file %s does not have attribute 'size' -- cannot check size",
                  path_name, file_name);
        return;
      }
      if (v != dat->size) {
        set_error("dat.size %lld in file %s and dim %d do not match", v, file_name, dat->dim);
        return;
      }
      if (!int_attr_of(*o, "dim", v)) {
        set_error("data set %s on file %s does not have attribute 'dim' -- cannot check dim",
                  path_name, file_name);
        return;
      }
      if (v != dat->dim) {
        set_error("dat.dim %lld in file %s and dim %d do not match", v, file_name, dat->dim);
        return;
      }
      const H::Attr *ta = o->attr("type");
      if (!ta || ta->type.cls != H::Cls::String) {
        set_error("data set %s on file %s does not have attribute 'type' -- cannot check type",
                  path_name, file_name);
        return;
      }
      if (!type_equivalent(ta->as_string(), dat->type)) {
        set_error("dat.type %s in file %s and type %s do not match", ta->as_string().c_str(),
                  file_name, dat->type);
        return;
      }
      if (o->dims != dims) {
        set_error("op_fetch_data_hdf5_file: dataset %s in file %s has another extent", path_name,
                  file_name);
        return;
      }
      // the dataset keeps its own type; the values are converted to it
      std::vector<uint8_t> conv(o->bytes());
      H::convert(t, buf.data(), o->type, conv.data(), o->count());
      o->mem = std::move(conv);
      o->store = H::Object::Store::Mem;
    } else {
      H::Object &n = f->put(path_name, t, dims, buf.data());
      n.set_attr(int_attr("size", dat->size));
      n.set_attr(int_attr("dim", dat->dim));
      n.set_attr(str_attr("type", dat->type, strlen(dat->type)));
    }
    f->save(file_name);
  } catch (const std::exception &e) {
    set_error("op_fetch_data_hdf5_file: %s: %s", file_name, e.what());
  }
}

void op_fetch_data_hdf5_file(op_dat dat, char const *file_name) {
  op_fetch_data_hdf5_file_path(dat, file_name, dat ? dat->name : nullptr);
}

// ---------------------------------------------------------------- op2b_h5_*

int op2b_h5_info(const char *file, const char *path, int *rank, long long dims[8], char *type,
                 int type_len) {
  try {
    auto f = H::File::open(file ? file : "");
    H::Object *o = f->find(path ? path : "");
    if (!o || o->group) return 1;
    if (o->dims.size() > 8) {
      set_error("op2b_h5_info: rank %zu above 8", o->dims.size());
      return -1;
    }
    if (rank) *rank = (int)o->dims.size();
    if (dims)
      for (size_t k = 0; k < o->dims.size(); k++) dims[k] = (long long)o->dims[k];
    if (type && type_len > 0) {
      std::string t = o->type.cls == H::Cls::String ? "string" : o->type.op2_name();
      snprintf(type, (size_t)type_len, "%s", t.c_str());
    }
    return 0;
  } catch (const std::exception &e) {
    set_error("op2b_h5_info: %s", e.what());
    return -1;
  }
}

int op2b_h5_read(const char *file, const char *path, const char *type, void *out,
                 long long count) {
  try {
    H::Type t;
    if (!type || !h5_type(type, t)) {
      set_error("op2b_h5_read: unknown type %s", type ? type : "(null)");
      return -1;
    }
    auto f = H::File::open(file ? file : "");
    H::Object *o = f->find(path ? path : "");
    if (!o || o->group) {
      set_error("op2b_h5_read: no dataset '%s' in %s", path ? path : "", file);
      return -1;
    }
    if ((long long)o->count() != count) {
      set_error("op2b_h5_read: dataset '%s' has %llu elements, not %lld", path,
                (unsigned long long)o->count(), count);
      return -1;
    }
    std::vector<uint8_t> v = f->read(*o, t);
    if (!v.empty()) memcpy(out, v.data(), v.size());
    return 0;
  } catch (const std::exception &e) {
    set_error("op2b_h5_read: %s", e.what());
    return -1;
  }
}

int op2b_h5_write(const char *file, const char *path, const char *type, int rank,
                  const long long *dims, const void *data) {
  try {
    H::Type t;
    if (!type || !h5_type(type, t) || rank < 0 || rank > 8 || (rank && !dims)) {
      set_error("op2b_h5_write: unknown type or bad rank");
      return -1;
    }
    std::vector<uint64_t> d(rank);
    for (int k = 0; k < rank; k++) {
      if (dims[k] < 0) {
        set_error("op2b_h5_write: negative extent");
        return -1;
      }
      d[k] = (uint64_t)dims[k];
    }
    auto f = file_exists(file) ? H::File::open(file) : H::File::create();
    f->put(path ? path : "", t, d, data);
    f->save(file);
    return 0;
  } catch (const std::exception &e) {
    set_error("op2b_h5_write: %s", e.what());
    return -1;
  }
}

int op2b_h5_set_attr(const char *file, const char *path, const char *name, const char *type,
                     int count, const void *data) {
  try {
    auto f = H::File::open(file ? file : "");
    H::Object *o = f->find(path ? path : "");
    if (!o || !name || !type || count < 0) {
      set_error("op2b_h5_set_attr: no object '%s' in %s, or no name or type", path ? path : "",
                file);
      return -1;
    }
    if (strcmp(type, "string") == 0) {
      std::string s = data ? (const char *)data : "";
      o->set_attr(str_attr(name, s, count > 0 ? (size_t)count : s.size()));
    } else {
      H::Attr a;
      a.name = name;
      if (!h5_type(type, a.type)) {
        set_error("op2b_h5_set_attr: unknown type %s", type);
        return -1;
      }
      a.dims = {(uint64_t)count};
      a.data.assign((const uint8_t *)data, (const uint8_t *)data + (size_t)count * a.type.size);
      o->set_attr(std::move(a));
    }
    f->save(file);
    return 0;
  } catch (const std::exception &e) {
    set_error("op2b_h5_set_attr: %s", e.what());
    return -1;
  }
}

// an attribute as text: a string's value, or numbers separated by spaces
int op2b_h5_get_attr(const char *file, const char *path, const char *name, char *out,
                     int out_len) {
  try {
    auto f = H::File::open(file ? file : "");
    H::Object *o = f->find(path ? path : "");
    const H::Attr *a = o && name ? o->attr(name) : nullptr;
    if (!a) return 1;
    std::string s;
    if (a->type.cls == H::Cls::String) {
      s = a->as_string();
    } else {
      std::vector<double> v(a->count());
      H::convert(a->type, a->data.data(), H::Type::real(8), v.data(), v.size());
      char b[40];
      for (size_t i = 0; i < v.size(); i++) {
        snprintf(b, sizeof b, i ? " %.17g" : "%.17g", v[i]);
        s += b;
      }
    }
    if (out && out_len > 0) snprintf(out, (size_t)out_len, "%s", s.c_str());
    return 0;
  } catch (const std::exception &e) {
    set_error("op2b_h5_get_attr: %s", e.what());
    return -1;
  }
}

// every object: "/path/" for a group, "/path" for a dataset, one a line;
// returns the bytes needed (with the terminating zero)
long long op2b_h5_list(const char *file, char *out, long long out_len) {
  try {
    auto f = H::File::open(file ? file : "");
    std::string s;
    struct Walk {
      std::string &s;
      void go(const H::Object &o, const std::string &p) {
        for (auto &c : o.children) {
          std::string q = p + "/" + c->name;
          s += c->group ? q + "/\n" : q + "\n";
          if (c->group) go(*c, q);
        }
      }
    } w{s};
    w.go(f->root(), "");
    if (out && out_len > 0) snprintf(out, (size_t)out_len, "%s", s.c_str());
    return (long long)s.size() + 1;
  } catch (const std::exception &e) {
    set_error("op2b_h5_list: %s", e.what());
    return -1;
  }
}

}  // extern "C"
