// HDF5 subset reader and writer (see h5file.h).  Structures and field orders
// follow the HDF5 File Format Specification: superblock (II.A), symbol table
// entries (III.C), v1 B-trees (III.A.1), symbol table nodes (III.B), local
// heaps (III.D), object headers (IV.A.1), and the header messages
// (IV.A.2): dataspace 0x0001, link info 0x0002, datatype 0x0003, fill value
// 0x0004/0x0005, link 0x0006, data layout 0x0008, filter pipeline 0x000B,
// attribute 0x000C, continuation 0x0010, symbol table 0x0011, attribute info
// 0x0015.
#include "h5file.h"

#include <sys/types.h>
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <cstring>
#include <set>

namespace op2b {
namespace h5 {

namespace {

constexpr uint8_t kSig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
constexpr int kInternalK = 16;     // group B-tree: 2K children a node
constexpr int kMinLeafK = 4;       // symbol table node: 2K entries
constexpr size_t kSte = 40;        // symbol table entry, 8-byte offsets and lengths
constexpr uint64_t kUndef = ~0ull;

[[noreturn]] void fail(const std::string &m) { throw Error(m); }

uint64_t undef_of(int n) { return n >= 8 ? ~0ull : ((1ull << (8 * n)) - 1); }
size_t pad8(size_t n) { return (n + 7) & ~(size_t)7; }

// little-endian cursor over a block of bytes
struct Cur {
  const uint8_t *p;
  size_t n, i = 0;
  Cur(const uint8_t *p_, size_t n_) : p(p_), n(n_) {}
  explicit Cur(const std::vector<uint8_t> &v) : p(v.data()), n(v.size()) {}
  void need(size_t k) const {
    if (k > n - i) fail("truncated structure in file");
  }
  uint64_t un(int k) {
    need(k);
    uint64_t v = 0;
    for (int j = 0; j < k; j++) v |= (uint64_t)p[i + j] << (8 * j);
    i += k;
    return v;
  }
  uint8_t u8() { return (uint8_t)un(1); }
  uint16_t u16() { return (uint16_t)un(2); }
  uint32_t u32() { return (uint32_t)un(4); }
  void skip(size_t k) {
    need(k);
    i += k;
  }
  const uint8_t *at() const { return p + i; }
  size_t left() const { return n - i; }
  bool sig(const char *s) {
    need(4);
    bool ok = memcmp(p + i, s, 4) == 0;
    i += 4;
    return ok;
  }
};

// byte sink
struct Out {
  std::vector<uint8_t> b;
  void u8(uint8_t v) { b.push_back(v); }
  void un(uint64_t v, int k) {
    for (int j = 0; j < k; j++) b.push_back((uint8_t)(v >> (8 * j)));
  }
  void u16(uint16_t v) { un(v, 2); }
  void u32(uint32_t v) { un(v, 4); }
  void u64(uint64_t v) { un(v, 8); }
  void raw(const void *p, size_t n) {
    const uint8_t *q = (const uint8_t *)p;
    b.insert(b.end(), q, q + n);
  }
  void str(const char *s) { raw(s, 4); }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  void align8() { b.resize(pad8(b.size()), 0); }
  void put_at(size_t pos, uint64_t v, int k) {
    for (int j = 0; j < k; j++) b[pos + j] = (uint8_t)(v >> (8 * j));
  }
  size_t size() const { return b.size(); }
};

// ---------------------------------------------------------------- datatypes

Type parse_type(Cur &c) {
  uint8_t cv = c.u8();
  int cls = cv & 15;
  uint8_t b0 = c.u8(), b1 = c.u8();
  c.u8();
  (void)b1;
  Type t;
  t.size = c.u32();
  switch (cls) {
    case 0: {
      t.cls = Cls::Fixed;
      t.big_endian = b0 & 1;
      t.is_signed = (b0 >> 3) & 1;
      uint16_t off = c.u16(), prec = c.u16();
      if (off != 0 || prec != 8 * t.size || t.size == 0 || t.size > 8)
        fail("fixed-point type with padding bits or of size " + std::to_string(t.size));
      break;
    }
    case 1: {
      t.cls = Cls::Float;
      if (b0 & 0x40) fail("VAX floating-point type");
      t.big_endian = b0 & 1;
      uint16_t off = c.u16(), prec = c.u16();
      uint8_t eloc = c.u8(), esz = c.u8(), mloc = c.u8(), msz = c.u8();
      uint32_t bias = c.u32();
      bool f64 = t.size == 8 && off == 0 && prec == 64 && eloc == 52 && esz == 11 &&
                 mloc == 0 && msz == 52 && bias == 1023;
      bool f32 = t.size == 4 && off == 0 && prec == 32 && eloc == 23 && esz == 8 &&
                 mloc == 0 && msz == 23 && bias == 127;
      if (!f64 && !f32) fail("floating-point type other than IEEE binary32 or binary64");
      break;
    }
    case 3:
      t.cls = Cls::String;
      t.str_pad = b0 & 15;
      if ((b0 >> 4) > 1) fail("string type of an unknown character set");
      break;
    default:
      fail("datatype class " + std::to_string(cls) + " is not supported");
  }
  return t;
}

void put_type(Out &o, const Type &t) {
  o.u8((uint8_t)(0x10 | (uint8_t)t.cls));  // version 1
  switch (t.cls) {
    case Cls::Fixed:
      o.u8((t.big_endian ? 1 : 0) | (t.is_signed ? 8 : 0));
      o.u8(0);
      o.u8(0);
      o.u32(t.size);
      o.u16(0);
      o.u16((uint16_t)(8 * t.size));
      break;
    case Cls::Float:
      // mantissa normalised with the leading one implied (bits 4-5 = 2),
      // sign bit the top bit
      o.u8((t.big_endian ? 1 : 0) | 0x20);
      o.u8((uint8_t)(8 * t.size - 1));
      o.u8(0);
      o.u32(t.size);
      o.u16(0);
      o.u16((uint16_t)(8 * t.size));
      if (t.size == 8) {
        o.u8(52), o.u8(11), o.u8(0), o.u8(52), o.u32(1023);
      } else {
        o.u8(23), o.u8(8), o.u8(0), o.u8(23), o.u32(127);
      }
      break;
    case Cls::String:
      o.u8(t.str_pad & 15);  // ASCII
      o.u8(0);
      o.u8(0);
      o.u32(t.size);
      break;
  }
}

// ---------------------------------------------------------------- dataspaces

void parse_space(Cur &c, int sl, std::vector<uint64_t> &dims) {
  uint8_t ver = c.u8(), rank = c.u8(), flags = c.u8();
  bool null = false;
  if (ver == 1) {
    c.skip(5);
  } else if (ver == 2) {
    null = c.u8() == 2;
  } else {
    fail("dataspace message version " + std::to_string(ver));
  }
  (void)flags;
  dims.resize(rank);
  for (auto &d : dims) d = c.un(sl);
  if (null) dims.assign(1, 0);  // no elements
}

void put_space(Out &o, const std::vector<uint64_t> &dims) {
  o.u8(1);  // version 1: rank 0 is a scalar
  o.u8((uint8_t)dims.size());
  o.u8(0);  // no maximum dimensions
  o.zeros(5);
  for (uint64_t d : dims) o.u64(d);
}

uint64_t count_of(const std::vector<uint64_t> &dims) {
  uint64_t n = 1;
  for (uint64_t d : dims) n *= d;
  return n;
}

// ---------------------------------------------------------------- number conversion

void load_bytes(const Type &t, const uint8_t *p, uint8_t *le) {
  if (t.big_endian)
    for (uint32_t j = 0; j < t.size; j++) le[j] = p[t.size - 1 - j];
  else
    memcpy(le, p, t.size);
}

void store_bytes(const Type &t, const uint8_t *le, uint8_t *p) {
  if (t.big_endian)
    for (uint32_t j = 0; j < t.size; j++) p[j] = le[t.size - 1 - j];
  else
    memcpy(p, le, t.size);
}

}  // namespace

Type Type::fixed(uint32_t bytes, bool sign) {
  Type t;
  t.cls = Cls::Fixed;
  t.size = bytes;
  t.is_signed = sign;
  return t;
}
Type Type::real(uint32_t bytes) {
  Type t;
  t.cls = Cls::Float;
  t.size = bytes;
  return t;
}
Type Type::str(uint32_t bytes) {
  Type t;
  t.cls = Cls::String;
  t.size = bytes;
  t.str_pad = 0;
  return t;
}

std::string Type::op2_name() const {
  if (big_endian) return "UNRECOGNISED";
  if (cls == Cls::Fixed && is_signed && size == 4) return "int";
  if (cls == Cls::Fixed && is_signed && size == 8) return "long";
  if (cls == Cls::Float && size == 4) return "float";
  if (cls == Cls::Float && size == 8) return "double";
  return "UNRECOGNISED";
}

void convert(const Type &from, const void *src, const Type &to, void *dst, uint64_t n) {
  const uint8_t *s = (const uint8_t *)src;
  uint8_t *d = (uint8_t *)dst;
  if (from.cls == Cls::String || to.cls == Cls::String) {
    if (from.cls != to.cls) fail("no conversion between strings and numbers");
    for (uint64_t i = 0; i < n; i++) {
      memset(d + i * to.size, to.str_pad == 2 ? ' ' : 0, to.size);
      memcpy(d + i * to.size, s + i * from.size, std::min(from.size, to.size));
    }
    return;
  }
  if (from.cls == to.cls && from.size == to.size && from.is_signed == to.is_signed &&
      from.big_endian == to.big_endian) {
    memcpy(d, s, n * from.size);
    return;
  }
  for (uint64_t i = 0; i < n; i++) {
    uint8_t le[8] = {0};
    load_bytes(from, s + i * from.size, le);
    bool is_real = from.cls == Cls::Float;
    double r = 0;
    int64_t v = 0;
    uint64_t u = 0;
    if (is_real) {
      if (from.size == 8) {
        memcpy(&r, le, 8);
      } else {
        float f;
        memcpy(&f, le, 4);
        r = f;
      }
    } else {
      memcpy(&u, le, 8);
      if (from.is_signed && from.size < 8 && (le[from.size - 1] & 0x80))
        u |= ~0ull << (8 * from.size);  // sign extension
      v = (int64_t)u;
    }
    uint8_t o[8] = {0};
    if (to.cls == Cls::Float) {
      double x = is_real ? r : (from.is_signed ? (double)v : (double)u);
      if (to.size == 8) {
        memcpy(o, &x, 8);
      } else {
        float f = (float)x;
        memcpy(o, &f, 4);
      }
    } else {
      // to integers: truncation toward zero, saturating at the type's range
      int bits = 8 * to.size;
      if (to.is_signed) {
        int64_t hi = bits == 64 ? INT64_MAX : (int64_t)((1ull << (bits - 1)) - 1);
        int64_t lo = -hi - 1;
        int64_t w;
        if (is_real)
          w = r != r ? 0 : r >= (double)hi ? hi : r <= (double)lo ? lo : (int64_t)r;
        else if (!from.is_signed && u > (uint64_t)hi)
          w = hi;
        else
          w = std::min(std::max(v, lo), hi);
        memcpy(o, &w, 8);
      } else {
        uint64_t hi = bits == 64 ? UINT64_MAX : ((1ull << bits) - 1);
        uint64_t w;
        if (is_real)
          w = !(r > 0) ? 0 : r >= (double)hi ? hi : (uint64_t)r;
        else if (from.is_signed && v < 0)
          w = 0;
        else
          w = std::min(u, hi);
        memcpy(o, &w, 8);
      }
    }
    store_bytes(to, o, d + i * to.size);
  }
}

uint64_t Attr::count() const { return count_of(dims); }

std::string Attr::as_string() const {
  if (type.cls != Cls::String) fail("attribute '" + name + "' is not a string");
  std::string s(data.begin(), data.end());
  if (type.str_pad == 2) {
    while (!s.empty() && s.back() == ' ') s.pop_back();
  } else {
    s = s.substr(0, strnlen(s.c_str(), s.size()));
  }
  return s;
}

uint64_t Object::count() const { return count_of(dims); }

Object *Object::child(const std::string &n) const {
  for (auto &c : children)
    if (c->name == n) return c.get();
  return nullptr;
}

const Attr *Object::attr(const std::string &n) const {
  for (auto &a : attrs)
    if (a.name == n) return &a;
  return nullptr;
}

void Object::set_attr(Attr a) {
  for (auto &x : attrs)
    if (x.name == a.name) {
      x = std::move(a);
      return;
    }
  attrs.push_back(std::move(a));
}

// ---------------------------------------------------------------- reading

struct File::Reader {
  File &f;
  std::set<uint64_t> seen;
  int depth = 0;

  explicit Reader(File &f_) : f(f_) {}

  std::vector<uint8_t> rd(uint64_t addr, size_t n) const {
    // sizes come from the file: bounded by it before anything is allocated
    if (n > f.fsize_ || addr > f.fsize_)
      fail("corrupt file: " + std::to_string(n) + " bytes at address " + std::to_string(addr) +
           " lie beyond its end");
    std::vector<uint8_t> v(n);
    if (n == 0) return v;
    if (addr == undef_of(f.sa_) || fseeko(f.fp_, (off_t)(f.base_ + addr), SEEK_SET) != 0 ||
        fread(v.data(), 1, n, f.fp_) != n)
      fail("truncated file: " + std::to_string(n) + " bytes at address " +
           std::to_string(addr) + " cannot be read");
    return v;
  }

  struct Msg {
    uint16_t type;
    uint8_t flags;
    std::vector<uint8_t> data;
  };

  // every message of the object header at addr, continuation blocks followed
  std::vector<Msg> messages(uint64_t addr) {
    std::vector<Msg> out;
    std::vector<uint8_t> head = rd(addr, 4);
    bool v2 = memcmp(head.data(), "OHDR", 4) == 0;
    struct Chunk {
      uint64_t addr, len;
    };
    std::vector<Chunk> todo;
    uint8_t ohflags = 0;
    if (!v2) {
      std::vector<uint8_t> p = rd(addr, 16);
      Cur c(p);
      if (c.u8() != 1) fail("object header version at address " + std::to_string(addr));
      c.skip(1 + 2 + 4);
      uint32_t size = c.u32();
      todo.push_back({addr + 16, size});
    } else {
      std::vector<uint8_t> p = rd(addr, 6);
      Cur c(p);
      c.skip(4);
      if (c.u8() != 2) fail("object header version at address " + std::to_string(addr));
      ohflags = c.u8();
      size_t pre = 6 + ((ohflags & 0x20) ? 16 : 0) + ((ohflags & 0x10) ? 4 : 0);
      int szb = 1 << (ohflags & 3);
      std::vector<uint8_t> q = rd(addr + pre, szb);
      Cur cq(q);
      uint64_t len = cq.un(szb);
      todo.push_back({addr + pre + szb, len});
    }
    for (size_t k = 0; k < todo.size(); k++) {
      if (todo.size() > 4096) fail("too many object header continuation blocks");
      Chunk ch = todo[k];
      std::vector<uint8_t> blk;
      size_t lo = 0, hi;
      if (!v2) {
        blk = rd(ch.addr, ch.len);
        hi = blk.size();
      } else if (k == 0) {
        blk = rd(ch.addr, ch.len);  // messages; the checksum follows
        hi = blk.size();
      } else {
        blk = rd(ch.addr, ch.len);
        if (blk.size() < 8 || memcmp(blk.data(), "OCHK", 4) != 0)
          fail("object header continuation block without its signature");
        lo = 4;
        hi = blk.size() - 4;
      }
      Cur c(blk.data(), hi);
      c.i = lo;
      size_t mh = v2 ? 4 + ((ohflags & 0x04) ? 2 : 0) : 8;
      while (c.left() >= mh) {
        Msg m;
        uint16_t len;
        if (!v2) {
          m.type = c.u16();
          len = c.u16();
          m.flags = c.u8();
          c.skip(3);
        } else {
          m.type = c.u8();
          len = c.u16();
          m.flags = c.u8();
          if (ohflags & 0x04) c.skip(2);
        }
        c.need(len);
        m.data.assign(c.at(), c.at() + len);
        c.skip(len);
        if (m.type == 0x10) {
          Cur d(m.data);
          uint64_t a = d.un(f.sa_), l = d.un(f.sl_);
          todo.push_back({a, l});
        } else if (m.type != 0) {
          out.push_back(std::move(m));
        }
      }
    }
    return out;
  }

  std::unique_ptr<Object> object(const std::string &name, uint64_t addr) {
    if (!seen.insert(addr).second)
      fail("object '" + name + "' is reached twice (hard links or a cycle): not supported");
    if (++depth > 64) fail("groups nested too deeply");
    std::vector<Msg> ms = messages(addr);
    auto o = std::make_unique<Object>();
    o->name = name;
    bool is_group = false, is_data = false;
    for (auto &m : ms) {
      if (m.type == 0x11 || m.type == 0x02 || m.type == 0x06) is_group = true;
      if (m.type == 0x08) is_data = true;
    }
    if (is_group) {
      o->group = true;
      for (auto &m : ms) {
        Cur c(m.data);
        if (m.type == 0x11) {
          uint64_t bt = c.un(f.sa_), hp = c.un(f.sa_);
          symbol_table(*o, bt, hp);
        } else if (m.type == 0x02) {
          c.skip(1);
          uint8_t fl = c.u8();
          if (fl & 1) c.skip(8);
          uint64_t heap = c.un(f.sa_);
          if (heap != undef_of(f.sa_))
            fail("group '" + name + "' keeps its links in dense storage: not supported");
        } else if (m.type == 0x06) {
          link(*o, c);
        }
      }
    } else if (is_data) {
      dataset(*o, ms);
    } else {
      o.reset();  // a committed datatype or another kind of object: skipped
      --depth;
      return o;
    }
    for (auto &m : ms) {
      if (m.type == 0x0C) {
        if (m.flags & 2) fail("shared attribute message: not supported");
        Cur c(m.data);
        o->attrs.push_back(attribute(c));
      } else if (m.type == 0x15) {
        Cur c(m.data);
        c.skip(1);
        uint8_t fl = c.u8();
        if (fl & 1) c.skip(2);
        uint64_t heap = c.un(f.sa_);
        if (heap != undef_of(f.sa_))
          fail("object '" + name + "' keeps its attributes in dense storage: not supported");
      }
    }
    --depth;
    return o;
  }

  void add_child(Object &g, std::unique_ptr<Object> c) {
    if (c) g.children.push_back(std::move(c));
  }

  void link(Object &g, Cur &c) {
    if (c.u8() != 1) fail("link message version");
    uint8_t fl = c.u8();
    uint8_t type = (fl & 0x08) ? c.u8() : 0;
    if (fl & 0x04) c.skip(8);
    if (fl & 0x10) c.skip(1);
    uint64_t nl = c.un(1 << (fl & 3));
    c.need(nl);
    std::string nm((const char *)c.at(), nl);
    c.skip(nl);
    if (type != 0) return;  // soft and external links are not followed
    uint64_t a = c.un(f.sa_);
    add_child(g, object(nm, a));
  }

  void symbol_table(Object &g, uint64_t btree, uint64_t heap) {
    std::vector<uint8_t> hh = rd(heap, 8 + 2 * f.sl_ + f.sa_);
    Cur c(hh);
    if (!c.sig("HEAP")) fail("local heap signature");
    c.skip(4);
    uint64_t dsize = c.un(f.sl_);
    c.un(f.sl_);
    uint64_t daddr = c.un(f.sa_);
    std::vector<uint8_t> names = rd(daddr, dsize);
    group_node(g, btree, names, 0);
  }

  void group_node(Object &g, uint64_t addr, const std::vector<uint8_t> &names, int lvl) {
    if (lvl > 32) fail("group B-tree too deep");
    size_t hsz = 8 + 2 * f.sa_;
    std::vector<uint8_t> h = rd(addr, hsz);
    Cur c(h);
    if (!c.sig("TREE")) fail("B-tree node signature");
    uint8_t type = c.u8(), level = c.u8();
    uint16_t n = c.u16();
    if (type != 0) fail("group B-tree of the wrong node type");
    std::vector<uint8_t> body = rd(addr + hsz, (size_t)n * (f.sl_ + f.sa_) + f.sl_);
    Cur b(body);
    b.un(f.sl_);
    for (int i = 0; i < n; i++) {
      uint64_t child = b.un(f.sa_);
      b.un(f.sl_);
      if (level > 0) {
        group_node(g, child, names, lvl + 1);
        continue;
      }
      std::vector<uint8_t> sh = rd(child, 8);
      Cur s(sh);
      if (!s.sig("SNOD")) fail("symbol table node signature");
      s.skip(2);
      uint16_t ns = s.u16();
      size_t ste = f.sl_ + f.sa_ + 24;
      std::vector<uint8_t> ents = rd(child + 8, ns * ste);
      Cur e(ents);
      for (int k = 0; k < ns; k++) {
        uint64_t off = e.un(f.sl_), oh = e.un(f.sa_);
        e.skip(24);
        if (off >= names.size()) fail("symbol name outside its heap");
        std::string nm((const char *)names.data() + off,
                       strnlen((const char *)names.data() + off, names.size() - off));
        add_child(g, object(nm, oh));
      }
    }
  }

  Attr attribute(Cur &c) {
    uint8_t ver = c.u8();
    uint8_t fl = c.u8();
    if (ver < 1 || ver > 3) fail("attribute message version");
    if (ver >= 2 && (fl & 3)) fail("attribute with a shared datatype or dataspace");
    uint16_t nl = c.u16(), tl = c.u16(), sl = c.u16();
    if (ver == 3) c.skip(1);
    auto pad = [&](size_t k) { return ver == 1 ? pad8(k) : k; };
    Attr a;
    c.need(nl);
    a.name.assign((const char *)c.at(), strnlen((const char *)c.at(), nl));
    c.skip(pad(nl));
    c.need(pad(tl));
    {
      Cur t(c.at(), tl);
      a.type = parse_type(t);
    }
    c.skip(pad(tl));
    c.need(pad(sl));
    {
      Cur s(c.at(), sl);
      parse_space(s, f.sl_, a.dims);
    }
    c.skip(pad(sl));
    uint64_t nb = a.count() * a.type.size;
    c.need(nb);
    a.data.assign(c.at(), c.at() + nb);
    c.skip(nb);
    return a;
  }

  void dataset(Object &o, const std::vector<Msg> &ms) {
    bool have_type = false, have_space = false;
    for (auto &m : ms) {
      Cur c(m.data);
      switch (m.type) {
        case 0x01:
          parse_space(c, f.sl_, o.dims);
          have_space = true;
          break;
        case 0x03:
          if (m.flags & 2) fail("dataset '" + o.name + "' has a committed datatype");
          o.type = parse_type(c);
          have_type = true;
          break;
        case 0x04: {
          uint32_t sz = c.u32();
          c.need(sz);
          if (o.fill.empty()) o.fill.assign(c.at(), c.at() + sz);
          break;
        }
        case 0x05: {
          uint8_t ver = c.u8();
          bool def;
          if (ver == 1 || ver == 2) {
            c.skip(2);
            def = c.u8() != 0 || ver == 1;
          } else {
            def = (c.u8() & 0x20) != 0;
          }
          if (def) {
            uint32_t sz = c.u32();
            c.need(sz);
            o.fill.assign(c.at(), c.at() + sz);
          }
          break;
        }
        case 0x08:
          layout(o, c);
          break;
        case 0x0B:
          pipeline(o, c);
          break;
        default:
          break;
      }
    }
    if (!have_type || !have_space) fail("dataset '" + o.name + "' without a datatype or dataspace");
    if (o.fill.size() != o.type.size) o.fill.clear();
  }

  void layout(Object &o, Cur &c) {
    uint8_t ver = c.u8();
    uint64_t un = undef_of(f.sa_);
    if (ver == 1 || ver == 2) {
      uint8_t nd = c.u8(), cls = c.u8();
      c.skip(5);
      uint64_t a = cls != 0 ? c.un(f.sa_) : 0;
      std::vector<uint32_t> d(nd);
      for (auto &x : d) x = c.u32();
      if (cls == 0) {
        uint32_t sz = c.u32();
        c.need(sz);
        o.mem.assign(c.at(), c.at() + sz);
        o.store = Object::Store::Mem;
      } else {
        o.addr = a;
        if (cls == 2) o.chunk = d;
        o.store = a == un ? Object::Store::Unallocated
                          : cls == 1 ? Object::Store::Contiguous : Object::Store::Chunked;
      }
    } else if (ver == 3 || ver == 4) {
      uint8_t cls = c.u8();
      if (cls == 0) {
        uint16_t sz = c.u16();
        c.need(sz);
        o.mem.assign(c.at(), c.at() + sz);
        o.store = Object::Store::Mem;
      } else if (cls == 1) {
        o.addr = c.un(f.sa_);
        o.store = o.addr == un ? Object::Store::Unallocated : Object::Store::Contiguous;
      } else if (cls == 2 && ver == 3) {
        uint8_t nd = c.u8();
        o.addr = c.un(f.sa_);
        o.chunk.resize(nd);
        for (auto &x : o.chunk) x = c.u32();
        o.store = o.addr == un ? Object::Store::Unallocated : Object::Store::Chunked;
      } else {
        fail("dataset '" + o.name + "': storage layout not supported (chunk indexes of layout "
             "version 4, virtual datasets)");
      }
    } else {
      fail("data layout message version " + std::to_string(ver));
    }
  }

  void pipeline(Object &o, Cur &c) {
    uint8_t ver = c.u8(), n = c.u8();
    if (ver == 1) c.skip(6);
    for (int k = 0; k < n; k++) {
      Object::Filter x;
      x.id = c.u16();
      uint16_t nl = (ver == 1 || x.id >= 256) ? c.u16() : 0;
      c.u16();
      uint16_t nv = c.u16();
      c.skip(ver == 1 ? pad8(nl) : nl);
      for (int j = 0; j < nv; j++) x.cd.push_back(c.u32());
      if (ver == 1 && (nv & 1)) c.skip(4);
      o.filters.push_back(x);
    }
  }
};

std::unique_ptr<File> File::create() {
  std::unique_ptr<File> f(new File());
  f->root_ = std::make_unique<Object>();
  f->root_->group = true;
  return f;
}

std::unique_ptr<File> File::open(const std::string &path) {
  std::unique_ptr<File> f(new File());
  f->fp_ = fopen(path.c_str(), "rb");
  if (!f->fp_) fail("cannot open file '" + path + "'");
  fseeko(f->fp_, 0, SEEK_END);
  uint64_t fsize = (uint64_t)ftello(f->fp_);
  f->fsize_ = fsize;
  // the superblock is at 0 or after a user block of 512, 1024, 2048, ... bytes
  uint64_t sb = kUndef;
  for (uint64_t off = 0; off + 8 <= fsize; off = off ? 2 * off : 512) {
    uint8_t s[8];
    fseeko(f->fp_, (off_t)off, SEEK_SET);
    if (fread(s, 1, 8, f->fp_) == 8 && memcmp(s, kSig, 8) == 0) {
      sb = off;
      break;
    }
  }
  if (sb == kUndef) fail("'" + path + "' is not an HDF5 file");
  std::vector<uint8_t> h(std::min<uint64_t>(fsize - sb, 256));
  fseeko(f->fp_, (off_t)sb, SEEK_SET);
  if (fread(h.data(), 1, h.size(), f->fp_) != h.size()) fail("cannot read the superblock");
  Cur c(h);
  c.skip(8);
  uint8_t ver = c.u8();
  uint64_t root_oh;
  if (ver <= 1) {
    c.skip(4);
    f->sa_ = c.u8();
    f->sl_ = c.u8();
    c.skip(1 + 4 + 4);
    if (ver == 1) c.skip(4);
  } else if (ver <= 3) {
    f->sa_ = c.u8();
    f->sl_ = c.u8();
    c.skip(1);
  } else {
    fail("superblock version " + std::to_string(ver) + " is not supported");
  }
  auto ok = [](int s) { return s == 2 || s == 4 || s == 8; };
  if (!ok(f->sa_) || !ok(f->sl_)) fail("sizes of offsets and lengths in the superblock");
  c.un(f->sa_);  // base address: addresses count from the superblock's position
  f->base_ = sb;
  if (ver <= 1) {
    c.un(f->sa_);  // free space
    c.un(f->sa_);  // end of file
    c.un(f->sa_);  // driver information
    c.un(f->sl_);  // root entry: link name offset
    root_oh = c.un(f->sa_);
  } else {
    c.un(f->sa_);  // superblock extension
    c.un(f->sa_);  // end of file
    root_oh = c.un(f->sa_);
  }
  Reader r(*f);
  f->root_ = r.object("", root_oh);
  if (!f->root_ || !f->root_->group) fail("the root object of '" + path + "' is not a group");
  return f;
}

File::~File() {
  if (fp_) fclose(fp_);
}

Object *File::find(const std::string &path) const {
  Object *o = root_.get();
  size_t i = 0;
  while (o && i < path.size()) {
    size_t j = path.find('/', i);
    if (j == std::string::npos) j = path.size();
    if (j > i) {
      if (!o->group) return nullptr;
      o = o->child(path.substr(i, j - i));
    }
    i = j + 1;
  }
  return o;
}

Object &File::put(const std::string &path, const Type &t, const std::vector<uint64_t> &dims,
                  const void *data) {
  std::vector<std::string> parts;
  for (size_t i = 0; i < path.size();) {
    size_t j = path.find('/', i);
    if (j == std::string::npos) j = path.size();
    if (j > i) parts.push_back(path.substr(i, j - i));
    i = j + 1;
  }
  if (parts.empty()) fail("empty dataset path");
  Object *g = root_.get();
  for (size_t k = 0; k + 1 < parts.size(); k++) {
    Object *c = g->child(parts[k]);
    if (!c) {
      auto n = std::make_unique<Object>();
      n->name = parts[k];
      n->group = true;
      c = n.get();
      g->children.push_back(std::move(n));
    } else if (!c->group) {
      fail("'" + parts[k] + "' in path '" + path + "' is a dataset, not a group");
    }
    g = c;
  }
  auto d = std::make_unique<Object>();
  d->name = parts.back();
  d->type = t;
  d->dims = dims;
  d->store = Object::Store::Mem;
  const uint8_t *p = (const uint8_t *)data;
  uint64_t nb = d->bytes();
  if (nb && !p) fail("no data for dataset '" + path + "'");
  d->mem.assign(p, p + nb);
  for (auto &c : g->children)
    if (c->name == d->name) {
      if (c->group) fail("'" + path + "' is a group");
      c = std::move(d);
      return *c;
    }
  g->children.push_back(std::move(d));
  return *g->children.back();
}

// ---------------------------------------------------------------- raw data

namespace {

std::vector<uint8_t> inflate_all(const std::vector<uint8_t> &in, size_t expect) {
  std::vector<uint8_t> out(expect);
  uLongf n = (uLongf)expect;
  int rc = uncompress(out.data(), &n, in.data(), (uLong)in.size());
  if (rc != Z_OK || n != expect) fail("a deflate-compressed chunk does not decompress");
  return out;
}

std::vector<uint8_t> unshuffle(const std::vector<uint8_t> &in, uint32_t es) {
  if (es <= 1) return in;
  std::vector<uint8_t> out(in.size());
  size_t n = in.size() / es;
  for (uint32_t b = 0; b < es; b++)
    for (size_t i = 0; i < n; i++) out[i * es + b] = in[b * n + i];
  // bytes left over past the whole elements are stored as they are
  std::copy(in.begin() + n * es, in.end(), out.begin() + n * es);
  return out;
}

}  // namespace

std::vector<uint8_t> File::read_raw(const Object &ds) const {
  if (ds.group) fail("'" + ds.name + "' is a group");
  uint64_t nb = ds.bytes();
  std::vector<uint8_t> out;
  auto filled = [&]() {
    std::vector<uint8_t> v(nb, 0);
    if (ds.fill.size() == ds.type.size && ds.type.size)
      for (uint64_t i = 0; i < ds.count(); i++)
        memcpy(v.data() + i * ds.type.size, ds.fill.data(), ds.type.size);
    return v;
  };
  Reader r(*const_cast<File *>(this));
  switch (ds.store) {
    case Object::Store::Mem:
      if (ds.mem.size() < nb) fail("compact dataset '" + ds.name + "' is shorter than its extent");
      return std::vector<uint8_t>(ds.mem.begin(), ds.mem.begin() + nb);
    case Object::Store::Unallocated:
      return filled();
    case Object::Store::Contiguous:
      return r.rd(ds.addr, nb);
    case Object::Store::Chunked:
      break;
  }
  // chunked: walk the chunk B-tree (node type 1)
  size_t rank = ds.dims.size();
  if (ds.chunk.size() != rank + 1 || rank == 0) fail("chunk dimensions of '" + ds.name + "'");
  uint32_t es = ds.chunk[rank];
  if (es != ds.type.size) fail("chunk element size of '" + ds.name + "'");
  uint64_t per = 1;
  for (size_t k = 0; k < rank; k++) per *= ds.chunk[k];
  out = filled();
  size_t ks = 8 + 8 * (rank + 1);
  std::vector<std::pair<uint64_t, int>> stack{{ds.addr, 0}};
  while (!stack.empty()) {
    auto [addr, lvl] = stack.back();
    stack.pop_back();
    if (lvl > 64) fail("chunk B-tree too deep");
    size_t hsz = 8 + 2 * sa_;
    std::vector<uint8_t> h = r.rd(addr, hsz);
    Cur c(h);
    if (!c.sig("TREE")) fail("chunk B-tree signature");
    uint8_t type = c.u8(), level = c.u8();
    uint16_t n = c.u16();
    if (type != 1) fail("chunk B-tree of the wrong node type");
    std::vector<uint8_t> body = r.rd(addr + hsz, (size_t)n * (ks + sa_) + ks);
    Cur b(body);
    for (int i = 0; i < n; i++) {
      uint32_t csize = b.u32(), mask = b.u32();
      std::vector<uint64_t> off(rank + 1);
      for (auto &x : off) x = b.un(8);
      uint64_t child = b.un(sa_);
      if (level > 0) {
        stack.push_back({child, lvl + 1});
        continue;
      }
      std::vector<uint8_t> data = r.rd(child, csize);
      for (int k = (int)ds.filters.size() - 1; k >= 0; k--) {
        if (mask & (1u << k)) continue;
        const auto &fl = ds.filters[k];
        if (fl.id == 1)
          data = inflate_all(data, per * es);
        else if (fl.id == 2)
          data = unshuffle(data, fl.cd.empty() ? es : fl.cd[0]);
        else if (fl.id == 3) {
          if (data.size() < 4) fail("fletcher32 chunk too short");
          data.resize(data.size() - 4);
        } else
          fail("dataset '" + ds.name + "' uses filter " + std::to_string(fl.id) +
               ": not supported");
      }
      if (data.size() < per * es) fail("chunk of '" + ds.name + "' shorter than its extent");
      // copy the chunk's rows that fall inside the dataset
      std::vector<uint64_t> idx(rank, 0);
      uint64_t last = ds.chunk[rank - 1];
      while (true) {
        bool inside = true;
        uint64_t g = 0;
        for (size_t k = 0; k + 1 < rank; k++) {
          uint64_t x = off[k] + idx[k];
          if (x >= ds.dims[k]) inside = false;
          g = g * ds.dims[k] + x;
        }
        if (inside && off[rank - 1] < ds.dims[rank - 1]) {
          uint64_t row0 = g * ds.dims[rank - 1] + off[rank - 1];
          uint64_t m = std::min<uint64_t>(last, ds.dims[rank - 1] - off[rank - 1]);
          uint64_t l = 0;
          for (size_t k = 0; k + 1 < rank; k++) l = l * ds.chunk[k] + idx[k];
          memcpy(out.data() + row0 * es, data.data() + l * last * es, m * es);
        }
        // next row of the chunk (all but the last dimension)
        int k = (int)rank - 2;
        for (; k >= 0; k--) {
          if (++idx[k] < ds.chunk[k]) break;
          idx[k] = 0;
        }
        if (k < 0) break;
      }
    }
  }
  return out;
}

std::vector<uint8_t> File::read(const Object &ds, const Type &to) const {
  std::vector<uint8_t> raw = read_raw(ds);
  std::vector<uint8_t> out(ds.count() * to.size);
  convert(ds.type, raw.data(), to, out.data(), ds.count());
  return out;
}

// ---------------------------------------------------------------- writing

namespace {

struct Writer {
  const File &src;
  Out o;
  int leaf_k = kMinLeafK;
  struct Place {
    const Object *ds;
    size_t patch;  // where the layout message's address goes
  };
  std::vector<Place> places;

  explicit Writer(const File &s) : src(s) {}

  static void msg(Out &oh, uint16_t type, uint8_t flags, const Out &data, int &count) {
    oh.u16(type);
    oh.u16((uint16_t)pad8(data.size()));
    oh.u8(flags);
    oh.zeros(3);
    oh.raw(data.b.data(), data.size());
    oh.align8();
    count++;
  }

  static Out attr_msg(const Attr &a) {
    Out t, s, m;
    put_type(t, a.type);
    put_space(s, a.dims);
    m.u8(1);
    m.u8(0);
    m.u16((uint16_t)(a.name.size() + 1));
    m.u16((uint16_t)t.size());
    m.u16((uint16_t)s.size());
    m.raw(a.name.c_str(), a.name.size() + 1);
    m.align8();
    m.raw(t.b.data(), t.size());
    m.align8();
    m.raw(s.b.data(), s.size());
    m.align8();
    if (a.data.size() != a.count() * a.type.size) fail("attribute '" + a.name + "' data size");
    m.raw(a.data.data(), a.data.size());
    return m;
  }

  // a version-1 object header holding `body` (messages); returns its address
  uint64_t header(const Out &body, int count) {
    o.align8();
    uint64_t at = o.size();
    o.u8(1);
    o.u8(0);
    o.u16((uint16_t)count);
    o.u32(1);
    o.u32((uint32_t)body.size());
    o.u32(0);
    o.raw(body.b.data(), body.size());
    return at;
  }

  uint64_t dataset(const Object &d) {
    Out body, m;
    int n = 0;
    put_space(m, d.dims);
    msg(body, 0x0001, 0, m, n);
    m = Out();
    put_type(m, d.type);
    msg(body, 0x0003, 1, m, n);
    m = Out();
    m.u8(2);  // fill value message version 2: allocated late, written if set, the
    m.u8(2);  // default (zero) value
    m.u8(2);
    m.u8(1);
    m.u32(0);
    msg(body, 0x0005, 1, m, n);
    m = Out();
    m.u8(3);  // layout version 3, contiguous
    m.u8(1);
    size_t addr_at = body.size() + 8 + 2;
    m.u64(kUndef);
    m.u64(d.bytes());
    msg(body, 0x0008, 1, m, n);
    for (auto &a : d.attrs) msg(body, 0x000C, 0, attr_msg(a), n);
    uint64_t at = header(body, n);
    if (d.bytes()) places.push_back({&d, (size_t)(at + 16 + addr_at)});
    return at;
  }

  struct GroupAddrs {
    uint64_t oh, btree, heap;
  };

  GroupAddrs group(const Object &g) {
    std::vector<const Object *> kids;
    for (auto &c : g.children) kids.push_back(c.get());
    std::sort(kids.begin(), kids.end(),
              [](const Object *a, const Object *b) { return strcmp(a->name.c_str(), b->name.c_str()) < 0; });
    for (size_t i = 1; i < kids.size(); i++)
      if (kids[i]->name == kids[i - 1]->name) fail("two objects named '" + kids[i]->name + "'");
    struct Ent {
      uint64_t name_off, oh;
      bool grp;
      uint64_t bt, hp;
    };
    std::vector<Ent> ents;
    Out heap;
    heap.zeros(8);  // offset 0: the empty name
    for (const Object *k : kids) {
      Ent e{};
      e.name_off = heap.size();
      heap.raw(k->name.c_str(), k->name.size() + 1);
      heap.align8();
      if (k->group) {
        GroupAddrs a = group(*k);
        e.oh = a.oh;
        e.grp = true;
        e.bt = a.btree;
        e.hp = a.heap;
      } else {
        e.oh = dataset(*k);
      }
      ents.push_back(e);
    }
    // local heap: header, then its data segment
    o.align8();
    GroupAddrs r{};
    r.heap = o.size();
    o.str("HEAP");
    o.u8(0);
    o.zeros(3);
    o.u64(heap.size());
    o.u64(1);  // no free block
    o.u64(r.heap + 32);
    o.raw(heap.b.data(), heap.size());
    // symbol table nodes of up to 2K entries each
    size_t per = 2 * (size_t)leaf_k;
    std::vector<uint64_t> snods, last;
    for (size_t s = 0; s < ents.size(); s += per) {
      o.align8();
      snods.push_back(o.size());
      size_t m = std::min(per, ents.size() - s);
      o.str("SNOD");
      o.u8(1);
      o.u8(0);
      o.u16((uint16_t)m);
      for (size_t k = s; k < s + m; k++) {
        const Ent &e = ents[k];
        o.u64(e.name_off);
        o.u64(e.oh);
        o.u32(e.grp ? 1 : 0);
        o.u32(0);
        if (e.grp) {
          o.u64(e.bt);
          o.u64(e.hp);
        } else {
          o.zeros(16);
        }
      }
      o.zeros((per - m) * kSte);
      last.push_back(ents[s + m - 1].name_off);
    }
    if (snods.size() > 2 * (size_t)kInternalK) fail("group too large");
    // one leaf B-tree node over the symbol table nodes
    o.align8();
    r.btree = o.size();
    o.str("TREE");
    o.u8(0);
    o.u8(0);
    o.u16((uint16_t)snods.size());
    o.u64(kUndef);
    o.u64(kUndef);
    o.u64(0);
    for (size_t i = 0; i < snods.size(); i++) {
      o.u64(snods[i]);
      o.u64(last[i]);
    }
    o.zeros((2 * kInternalK - snods.size()) * 16);
    Out body, m;
    int n = 0;
    m.u64(r.btree);
    m.u64(r.heap);
    msg(body, 0x0011, 1, m, n);
    for (auto &a : g.attrs) msg(body, 0x000C, 0, attr_msg(a), n);
    r.oh = header(body, n);
    return r;
  }

  static size_t max_children(const Object &g) {
    size_t m = g.children.size();
    for (auto &c : g.children)
      if (c->group) m = std::max(m, max_children(*c));
    return m;
  }
};

}  // namespace

void File::save(const std::string &path) const {
  Writer w(*this);
  size_t mc = Writer::max_children(*root_);
  // a group's entries fill at most 2 * kInternalK symbol table nodes of
  // 2 * leaf_k entries each
  w.leaf_k = (int)std::max<size_t>(kMinLeafK, (mc + 4 * kInternalK - 1) / (4 * kInternalK));
  if (w.leaf_k > 32767) fail("group too large");
  // superblock version 0, patched at the end
  Out &o = w.o;
  o.raw(kSig, 8);
  o.u8(0), o.u8(0), o.u8(0), o.u8(0), o.u8(0), o.u8(8), o.u8(8), o.u8(0);
  o.u16((uint16_t)w.leaf_k);
  o.u16(kInternalK);
  o.u32(0);
  o.u64(0);       // base address
  o.u64(kUndef);  // free space
  size_t eof_at = o.size();
  o.u64(0);       // end of file
  o.u64(kUndef);  // driver information
  size_t root_at = o.size();
  o.zeros(kSte);
  Writer::GroupAddrs ra = w.group(*root_);
  {
    Out e;
    e.u64(0);
    e.u64(ra.oh);
    e.u32(1);
    e.u32(0);
    e.u64(ra.btree);
    e.u64(ra.heap);
    memcpy(o.b.data() + root_at, e.b.data(), kSte);
  }
  o.align8();
  uint64_t at = o.size();
  for (auto &p : w.places) {
    o.put_at(p.patch, at, 8);
    at = pad8(at + p.ds->bytes());
  }
  o.put_at(eof_at, at, 8);
  std::string tmp = path + ".tmp" + std::to_string((long)getpid());
  FILE *fp = fopen(tmp.c_str(), "wb");
  if (!fp) fail("cannot create '" + tmp + "'");
  bool ok = fwrite(o.b.data(), 1, o.size(), fp) == o.size();
  uint64_t pos = o.size();
  static const uint8_t zero[8] = {0};
  for (auto &p : w.places) {
    if (!ok) break;
    std::vector<uint8_t> tmpbuf;
    const std::vector<uint8_t> *data = &p.ds->mem;
    if (p.ds->store != Object::Store::Mem || p.ds->mem.size() != p.ds->bytes()) {
      tmpbuf = read_raw(*p.ds);
      data = &tmpbuf;
    }
    ok = fwrite(data->data(), 1, p.ds->bytes(), fp) == p.ds->bytes();
    pos += p.ds->bytes();
    size_t gap = pad8(pos) - pos;
    if (ok && gap) ok = fwrite(zero, 1, gap, fp) == gap;
    pos += gap;
  }
  ok = (fclose(fp) == 0) && ok;
  if (!ok || rename(tmp.c_str(), path.c_str()) != 0) {
    remove(tmp.c_str());
    fail("cannot write '" + path + "'");
  }
}

}  // namespace h5
}  // namespace op2b
