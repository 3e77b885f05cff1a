// h5io.cpp - checkpoint files in the reference's HDF5 layout, read and written without an HDF5
// library.
//
// The reference keeps its restart and field files through parallel HDF5 (channel_hdf5_io,
// module_hdf5_io.f90:6-456; data_store.f90:11-173 writes them, initial_step.f90:184-423 reads
// them).  Every dataset sits in the root group:
//   lines   1-D float64 (or int32 for timestep, nx, ny, nz, LABS_K, LABS_BW) of length n,
//   planes  2-D float64, Fortran (a, b) stored as C dims (b, a),
//   fields  3-D, Fortran (ny, nx/2, nz) stored as C dims (nz, nx/2, ny), each element an HDF5
//           array of two float64 (re, im) -- "ESIO layout 0" (module_hdf5_io.f90:3-5);
// string attributes on the root group (io_string_set, :169-210) and optional dataset comments.
// Files written by the older ESIO library carry an int32[8] attribute `esio_field_metadata` on
// each field; its 4th entry is the layout (0, 1 or 2; 2 flattens the field to (nz * nx/2, ny)),
// entries 5..7 the dimensions (nz, nx/2, ny) and the 8th the components (:313-345).
//
// What is implemented is the part of the HDF5 file format (version 0 superblock) those files use,
// as the HDF5 library writes it with its default settings:
//   superblock version 0, 8-byte offsets and lengths;
//   the root group as a symbol table: a version-1 B-tree of group nodes (signature TREE) over
//   symbol-table nodes (SNOD) and a local heap (HEAP) of link names;
//   version-1 object headers with continuation blocks;
//   dataspace (versions 1, 2), datatype (fixed-point, IEEE float, string, array versions 2, 3),
//   data layout (versions 1-3; contiguous and compact storage), attribute (versions 1-3),
//   comment and modification-time messages.
// Chunked or compressed storage, version-2 object headers and version-2/3 superblocks are
// refused with an error naming them.  The reader checks every address against the file size.
//
// A writer builds the whole file in one pass when it is closed: superblock, root object header,
// local heap, one B-tree node over at most 32 symbol-table nodes of up to 8 names (the
// superblock's group K values 16 and 4), dataset object headers, then the raw data, with
// datasets in creation order and links sorted by name as the B-tree requires.  A file opened for
// update is read whole and written again on close (the reference's rank-0 statistics append).
//
// The checks a read makes, and their messages, follow transfer() and legacy_layout()
// (module_hdf5_io.f90:212-311, 313-345): rank, dimensions, array class and component count, base
// type class and size, and the legacy metadata.  The reference aborts on them; here they return
// KMM_ERR_IO with the same text.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "kmm_internal.h"

namespace kmm {
namespace h5 {
namespace {

constexpr uint64_t kUndef = ~0ull;

struct Error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

[[noreturn]] void fail(const std::string &m) { throw Error(m); }

// ---------------------------------------------------------------------------------------------
// In-memory model

enum Cls { kFixed = 0, kFloat = 1, kString = 3, kArray = 10 };

struct Type {
  int cls = kFloat;
  uint32_t size = 8;
  bool big = false;       // byte order
  bool sgn = true;        // fixed-point sign
  std::vector<uint32_t> adims;  // array dimensions
  std::shared_ptr<Type> base;   // array base type
  int array_version = 2;
};

Type f64() { return Type{}; }
Type i32() {
  Type t;
  t.cls = kFixed;
  t.size = 4;
  return t;
}
Type f64_array(uint32_t n) {
  Type t;
  t.cls = kArray;
  t.size = 8 * n;
  t.adims = {n};
  t.base = std::make_shared<Type>(f64());
  return t;
}
Type str_type(uint32_t n) {
  Type t;
  t.cls = kString;
  t.size = n;
  return t;
}

struct Attr {
  std::string name;
  Type type;
  bool scalar = true;
  std::vector<uint64_t> dims;
  std::vector<uint8_t> data;
};

struct Dataset {
  std::string name;
  std::vector<uint64_t> dims;
  Type type;
  std::vector<uint8_t> data;  // stored bytes, in the type's byte order
  std::string comment;
  std::vector<Attr> attrs;
  const Attr *attr(const std::string &n) const {
    for (const Attr &a : attrs)
      if (a.name == n) return &a;
    return nullptr;
  }
  uint64_t elements() const {
    uint64_t n = 1;
    for (uint64_t d : dims) n *= d;
    return n;
  }
};

struct Model {
  std::vector<Attr> root_attrs;
  std::vector<Dataset> sets;
  Dataset *find(const std::string &n) {
    for (Dataset &d : sets)
      if (d.name == n) return &d;
    return nullptr;
  }
};

// ---------------------------------------------------------------------------------------------
// Reader

struct Bytes {
  const std::vector<uint8_t> &b;
  void need(uint64_t off, uint64_t n) const {
    if (off > b.size() || n > b.size() - off) fail("malformed HDF5 file: address past the end of the file");
  }
  uint64_t u(uint64_t off, int n) const {
    need(off, n);
    uint64_t v = 0;
    for (int i = n - 1; i >= 0; --i) v = (v << 8) | b[off + i];
    return v;
  }
  uint8_t u8(uint64_t o) const { return (uint8_t)u(o, 1); }
  uint16_t u16(uint64_t o) const { return (uint16_t)u(o, 2); }
  uint32_t u32(uint64_t o) const { return (uint32_t)u(o, 4); }
  uint64_t u64(uint64_t o) const { return u(o, 8); }
  bool sig(uint64_t o, const char *s) const {
    need(o, 4);
    return std::memcmp(&b[o], s, 4) == 0;
  }
  std::string cstr(uint64_t o) const {
    std::string s;
    for (;; ++o) {
      need(o, 1);
      if (!b[o]) return s;
      s.push_back((char)b[o]);
    }
  }
};

struct Msg {
  uint16_t type;
  uint64_t off, size;
};

// (datatype, bytes it took)
Type parse_type(const Bytes &B, uint64_t o, uint64_t avail, uint64_t *used) {
  if (avail < 8) fail("malformed HDF5 datatype message");
  Type t;
  const uint8_t cv = B.u8(o);
  const int ver = cv >> 4;
  t.cls = cv & 15;
  const uint32_t bits = (uint32_t)B.u(o + 1, 3);
  t.size = B.u32(o + 4);
  uint64_t n = 8;
  switch (t.cls) {
    case kFixed:
      t.big = bits & 1;
      t.sgn = (bits >> 3) & 1;
      if (B.u16(o + 8) != 0 || B.u16(o + 10) != 8 * t.size) fail("unsupported HDF5 integer type (padding bits)");
      n += 4;
      break;
    case kFloat: {
      t.big = bits & 1;
      if (bits & 0x40) fail("unsupported HDF5 float byte order (VAX)");
      const int eloc = B.u8(o + 12), esz = B.u8(o + 13), mloc = B.u8(o + 14), msz = B.u8(o + 15);
      const uint32_t bias = B.u32(o + 16);
      const bool ieee8 = t.size == 8 && eloc == 52 && esz == 11 && mloc == 0 && msz == 52 && bias == 1023;
      const bool ieee4 = t.size == 4 && eloc == 23 && esz == 8 && mloc == 0 && msz == 23 && bias == 127;
      if (B.u16(o + 8) != 0 || !(ieee8 || ieee4)) fail("unsupported HDF5 float type (not IEEE binary32/64)");
      n += 12;
      break;
    }
    case kString:
      break;
    case kArray: {
      const int nd = B.u8(o + 8);
      t.array_version = ver;
      uint64_t p = o + (ver == 2 ? 12 : 9);
      for (int i = 0; i < nd; ++i, p += 4) t.adims.push_back(B.u32(p));
      if (ver == 2) p += 4 * (uint64_t)nd;  // permutation indices
      uint64_t bu = 0;
      t.base = std::make_shared<Type>(parse_type(B, p, avail - (p - o), &bu));
      n = (p - o) + bu;
      break;
    }
    default:
      fail("unsupported HDF5 datatype class " + std::to_string(t.cls));
  }
  if (n > avail) fail("malformed HDF5 datatype message");
  *used = n;
  return t;
}

// dims (scalar: empty with *scalar = true)
std::vector<uint64_t> parse_space(const Bytes &B, uint64_t o, bool *scalar) {
  const int ver = B.u8(o), nd = B.u8(o + 1);
  uint64_t p;
  if (ver == 1) {
    p = o + 8;
    *scalar = nd == 0;
  } else if (ver == 2) {
    const int kind = B.u8(o + 3);
    if (kind == 2) fail("unsupported HDF5 null dataspace");
    *scalar = kind == 0;
    p = o + 4;
  } else {
    fail("unsupported HDF5 dataspace version " + std::to_string(ver));
  }
  std::vector<uint64_t> d;
  for (int i = 0; i < nd; ++i) d.push_back(B.u64(p + 8 * (uint64_t)i));
  return d;
}

std::vector<Msg> object_messages(const Bytes &B, uint64_t addr) {
  if (B.sig(addr, "OHDR")) fail("unsupported HDF5 object header version 2");
  if (B.u8(addr) != 1) fail("unsupported HDF5 object header version " + std::to_string(B.u8(addr)));
  const uint32_t nmsg = B.u16(addr + 2);
  const uint32_t hsize = B.u32(addr + 8);
  std::vector<std::pair<uint64_t, uint64_t>> blocks{{addr + 16, hsize}};
  std::vector<Msg> out;
  for (size_t k = 0; k < blocks.size() && out.size() < nmsg; ++k) {
    uint64_t p = blocks[k].first;
    const uint64_t end = p + blocks[k].second;
    B.need(p, blocks[k].second);
    while (p + 8 <= end && out.size() < nmsg) {
      Msg m{B.u16(p), p + 8, B.u16(p + 2)};
      if (m.off + m.size > end) fail("malformed HDF5 object header");
      if (B.u8(p + 4) & 2) fail("unsupported shared HDF5 message");
      if (m.type == 0x10) blocks.push_back({B.u64(m.off), B.u64(m.off + 8)});
      out.push_back(m);
      p = m.off + m.size;
    }
    if (blocks.size() > 1024) fail("malformed HDF5 object header (continuations)");
  }
  return out;
}

uint64_t pad8(uint64_t n) { return (n + 7) & ~7ull; }

Attr parse_attr(const Bytes &B, const Msg &m) {
  const uint64_t o = m.off;
  const int ver = B.u8(o);
  const uint16_t nl = B.u16(o + 2), tl = B.u16(o + 4), sl = B.u16(o + 6);
  uint64_t p = o + (ver == 3 ? 9 : 8);
  if (ver < 1 || ver > 3) fail("unsupported HDF5 attribute version " + std::to_string(ver));
  auto adv = [&](uint64_t n) { return ver == 1 ? pad8(n) : n; };
  Attr a;
  B.need(p, nl);
  a.name = B.cstr(p);
  p += adv(nl);
  uint64_t used = 0;
  a.type = parse_type(B, p, tl, &used);
  p += adv(tl);
  a.dims = parse_space(B, p, &a.scalar);
  p += adv(sl);
  uint64_t ne = 1;
  for (uint64_t d : a.dims) ne *= d;
  const uint64_t nb = ne * a.type.size;
  if (p + nb > m.off + m.size) fail("malformed HDF5 attribute " + a.name);
  a.data.assign(B.b.begin() + (long)p, B.b.begin() + (long)(p + nb));
  return a;
}

void read_dataset(const Bytes &B, uint64_t addr, Dataset &d) {
  bool have_space = false, have_type = false, have_layout = false, scalar = false;
  uint64_t daddr = kUndef, dsize = 0;
  const uint8_t *compact = nullptr;
  for (const Msg &m : object_messages(B, addr)) {
    switch (m.type) {
      case 0x01:
        d.dims = parse_space(B, m.off, &scalar);
        have_space = true;
        break;
      case 0x03: {
        uint64_t used = 0;
        d.type = parse_type(B, m.off, m.size, &used);
        have_type = true;
        break;
      }
      case 0x08: {
        const int ver = B.u8(m.off);
        if (ver == 3) {
          const int cls = B.u8(m.off + 1);
          if (cls == 0) {
            dsize = B.u16(m.off + 2);
            B.need(m.off + 4, dsize);
            compact = &B.b[m.off + 4];
          } else if (cls == 1) {
            daddr = B.u64(m.off + 2);
            dsize = B.u64(m.off + 10);
          } else {
            fail("unsupported HDF5 storage (chunked or virtual) for dataset " + d.name);
          }
        } else if (ver == 1 || ver == 2) {
          const int nd = B.u8(m.off + 1), cls = B.u8(m.off + 2);
          uint64_t p = m.off + 8;
          if (cls == 1) {
            daddr = B.u64(p);
            p += 8;
          } else if (cls != 0) {
            fail("unsupported HDF5 storage (chunked) for dataset " + d.name);
          }
          uint64_t n = 1;
          for (int i = 0; i < nd; ++i) n *= B.u32(p + 4 * (uint64_t)i);
          p += 4 * (uint64_t)nd;
          if (cls == 0) {
            dsize = B.u32(p);
            B.need(p + 4, dsize);
            compact = &B.b[p + 4];
          } else {
            dsize = n;
          }
        } else {
          fail("unsupported HDF5 layout message version " + std::to_string(ver));
        }
        have_layout = true;
        break;
      }
      case 0x0C:
        d.attrs.push_back(parse_attr(B, m));
        break;
      case 0x0D:
        d.comment = B.cstr(m.off);
        break;
      default:
        break;
    }
  }
  if (!have_space || !have_type || !have_layout) fail("malformed HDF5 dataset " + d.name);
  if (scalar) d.dims.clear();
  const uint64_t nb = d.elements() * d.type.size;
  if (compact) {
    if (dsize < nb) fail("malformed HDF5 dataset " + d.name);
    d.data.assign(compact, compact + nb);
  } else if (daddr == kUndef) {
    d.data.assign(nb, 0);  // never written: the default fill value
  } else {
    if (dsize < nb) fail("malformed HDF5 dataset " + d.name);
    B.need(daddr, nb);
    d.data.assign(B.b.begin() + (long)daddr, B.b.begin() + (long)(daddr + nb));
  }
}

void walk_group_btree(const Bytes &B, uint64_t node, uint64_t heap_data, int depth,
                      std::vector<std::pair<std::string, uint64_t>> &links) {
  if (depth > 64) fail("malformed HDF5 group B-tree");
  if (!B.sig(node, "TREE") || B.u8(node + 4) != 0) fail("malformed HDF5 group B-tree");
  const int level = B.u8(node + 5);
  const int used = B.u16(node + 6);
  for (int i = 0; i < used; ++i) {
    const uint64_t child = B.u64(node + 24 + 8 + 16 * (uint64_t)i);
    if (level > 0) {
      walk_group_btree(B, child, heap_data, depth + 1, links);
      continue;
    }
    if (!B.sig(child, "SNOD") || B.u8(child + 4) != 1) fail("malformed HDF5 symbol table node");
    const int nsym = B.u16(child + 6);
    for (int s = 0; s < nsym; ++s) {
      const uint64_t e = child + 8 + 40 * (uint64_t)s;
      const uint32_t cache = B.u32(e + 16);
      if (cache == 1) continue;  // a subgroup: the reference keeps everything in the root group
      links.push_back({B.cstr(heap_data + B.u64(e)), B.u64(e + 8)});
    }
  }
}

Model read_model(const std::vector<uint8_t> &bytes) {
  const Bytes B{bytes};
  static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  if (bytes.size() < 96 || std::memcmp(bytes.data(), sig, 8) != 0) fail("not an HDF5 file");
  if (B.u8(8) != 0) fail("unsupported HDF5 superblock version " + std::to_string(B.u8(8)));
  if (B.u8(13) != 8 || B.u8(14) != 8) fail("unsupported HDF5 offset or length size");
  if (B.u64(24) != 0) fail("unsupported HDF5 base address");
  const uint64_t root = B.u64(56 + 8);
  Model M;
  uint64_t btree = kUndef, heap = kUndef;
  for (const Msg &m : object_messages(B, root)) {
    if (m.type == 0x11) {
      btree = B.u64(m.off);
      heap = B.u64(m.off + 8);
    } else if (m.type == 0x0C) {
      M.root_attrs.push_back(parse_attr(B, m));
    }
  }
  if (btree == kUndef || heap == kUndef) fail("unsupported HDF5 root group (no symbol table)");
  if (!B.sig(heap, "HEAP")) fail("malformed HDF5 local heap");
  const uint64_t heap_data = B.u64(heap + 24);
  std::vector<std::pair<std::string, uint64_t>> links;
  walk_group_btree(B, btree, heap_data, 0, links);
  for (const auto &l : links) {
    Dataset d;
    d.name = l.first;
    read_dataset(B, l.second, d);
    M.sets.push_back(std::move(d));
  }
  return M;
}

// ---------------------------------------------------------------------------------------------
// Writer

struct Out {
  std::vector<uint8_t> b;
  void put(uint64_t v, int n) {
    for (int i = 0; i < n; ++i) b.push_back((uint8_t)(v >> (8 * i)));
  }
  void bytes(const void *p, size_t n) {
    const uint8_t *c = static_cast<const uint8_t *>(p);
    b.insert(b.end(), c, c + n);
  }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  void align8() { zeros(pad8(b.size()) - b.size()); }
};

void put_type(Out &o, const Type &t) {
  const uint32_t bits = t.cls == kFixed ? ((t.big ? 1u : 0u) | (t.sgn ? 8u : 0u))
                        : t.cls == kFloat ? ((t.big ? 1u : 0u) | 0x20u | (uint32_t)(8 * t.size - 1) << 8)
                                          : 0u;
  const int ver = t.cls == kArray ? t.array_version : 1;
  o.put((uint64_t)(ver << 4 | t.cls), 1);
  o.put(bits, 3);
  o.put(t.size, 4);
  if (t.cls == kFixed) {
    o.put(0, 2);
    o.put(8 * t.size, 2);
  } else if (t.cls == kFloat) {
    o.put(0, 2);
    o.put(8 * t.size, 2);
    if (t.size == 8) {
      o.put(52, 1), o.put(11, 1), o.put(0, 1), o.put(52, 1), o.put(1023, 4);
    } else {
      o.put(23, 1), o.put(8, 1), o.put(0, 1), o.put(23, 1), o.put(127, 4);
    }
  } else if (t.cls == kArray) {
    o.put(t.adims.size(), 1);
    if (t.array_version == 2) o.zeros(3);
    for (uint32_t d : t.adims) o.put(d, 4);
    if (t.array_version == 2)
      for (size_t i = 0; i < t.adims.size(); ++i) o.put(i, 4);
    put_type(o, *t.base);
  }
}

void put_space(Out &o, bool scalar, const std::vector<uint64_t> &dims) {
  o.put(1, 1);
  o.put(scalar ? 0 : dims.size(), 1);
  o.put(scalar ? 0 : 1, 1);  // maximum dimensions present (equal to the dimensions)
  o.zeros(5);
  if (scalar) return;
  for (uint64_t d : dims) o.put(d, 8);
  for (uint64_t d : dims) o.put(d, 8);
}

std::vector<uint8_t> serial(void (*fn)(Out &, const void *), const void *arg) {
  Out o;
  fn(o, arg);
  return o.b;
}

struct MsgOut {
  uint16_t type;
  uint8_t flags;
  std::vector<uint8_t> body;  // padded to 8
};

MsgOut msg(uint16_t type, uint8_t flags, std::vector<uint8_t> body) {
  body.resize(pad8(body.size()), 0);
  return MsgOut{type, flags, std::move(body)};
}

MsgOut attr_msg(const Attr &a) {
  Out t, s;
  put_type(t, a.type);
  put_space(s, a.scalar, a.dims);
  Out o;
  o.put(1, 1);
  o.put(0, 1);
  o.put(a.name.size() + 1, 2);
  o.put(t.b.size(), 2);
  o.put(s.b.size(), 2);
  o.bytes(a.name.c_str(), a.name.size() + 1);
  o.align8();
  o.bytes(t.b.data(), t.b.size());
  o.align8();
  o.bytes(s.b.data(), s.b.size());
  o.align8();
  o.bytes(a.data.data(), a.data.size());
  return msg(0x0C, 0, o.b);
}

uint64_t header_size(const std::vector<MsgOut> &ms) {
  uint64_t n = 0;
  for (const MsgOut &m : ms) n += 8 + m.body.size();
  return n;
}

void put_header(Out &o, const std::vector<MsgOut> &ms) {
  o.put(1, 1);
  o.put(0, 1);
  o.put(ms.size(), 2);
  o.put(1, 4);
  o.put(header_size(ms), 4);
  o.zeros(4);
  for (const MsgOut &m : ms) {
    o.put(m.type, 2);
    o.put(m.body.size(), 2);
    o.put(m.flags, 1);
    o.zeros(3);
    o.bytes(m.body.data(), m.body.size());
  }
}

std::vector<uint8_t> write_model(const Model &M) {
  constexpr int kLeafK = 4, kNodeK = 16;
  const size_t n = M.sets.size();
  // links sorted by name, split over symbol-table nodes of at most 2 * kLeafK names
  std::vector<size_t> order(n);
  for (size_t i = 0; i < n; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return M.sets[a].name < M.sets[b].name; });
  const size_t nsnod = std::max<size_t>(1, (n + 2 * kLeafK - 1) / (2 * kLeafK));
  if (nsnod > 2 * kNodeK) fail("too many datasets for one group node (256 at most)");
  // local heap: "" at 0, then every name, 8-byte padded, then one free block (offset of the
  // next free block, 1 = none, and its size) as the HDF5 library leaves at a heap's end
  std::vector<uint64_t> name_off(n);
  Out heapd;
  heapd.zeros(8);
  for (size_t i = 0; i < n; ++i) {
    name_off[i] = heapd.b.size();
    heapd.bytes(M.sets[i].name.c_str(), M.sets[i].name.size() + 1);
    heapd.align8();
  }
  const uint64_t heap_free = heapd.b.size();
  heapd.put(1, 8);
  heapd.put(16, 8);
  // per-dataset headers (data addresses patched below)
  const uint32_t now = (uint32_t)std::time(nullptr);
  std::vector<std::vector<MsgOut>> dh(n);
  for (size_t i = 0; i < n; ++i) {
    const Dataset &d = M.sets[i];
    Out s, t, f, mt;
    put_space(s, d.dims.empty(), d.dims);
    put_type(t, d.type);
    // fill value, version 2: allocation time early, write time if set, value defined, size 0
    f.put(2, 1), f.put(1, 1), f.put(2, 1), f.put(1, 1), f.put(0, 4);
    mt.put(1, 1), mt.zeros(3), mt.put(now, 4);
    dh[i].push_back(msg(0x01, 0, s.b));
    dh[i].push_back(msg(0x03, 1, t.b));
    dh[i].push_back(msg(0x05, 1, f.b));
    dh[i].push_back(msg(0x08, 1, std::vector<uint8_t>(18, 0)));  // layout placeholder
    dh[i].push_back(msg(0x12, 0, mt.b));
    if (!d.comment.empty()) {
      std::vector<uint8_t> c(d.comment.begin(), d.comment.end());
      c.push_back(0);
      dh[i].push_back(msg(0x0D, 0, c));
    }
    for (const Attr &a : d.attrs) dh[i].push_back(attr_msg(a));
  }
  std::vector<MsgOut> rh;
  rh.push_back(msg(0x11, 0, std::vector<uint8_t>(16, 0)));  // symbol table placeholder
  for (const Attr &a : M.root_attrs) rh.push_back(attr_msg(a));
  // addresses
  const uint64_t a_root = 96;
  const uint64_t a_heap = a_root + 16 + header_size(rh);
  const uint64_t a_heapd = a_heap + 32;
  const uint64_t a_tree = a_heapd + heapd.b.size();
  const uint64_t tree_size = 24 + (2 * kNodeK + 1) * 8 + 2 * kNodeK * 8;
  const uint64_t snod_size = 8 + 2 * kLeafK * 40;
  const uint64_t a_snod = a_tree + tree_size;
  uint64_t p = a_snod + nsnod * snod_size;
  std::vector<uint64_t> a_dh(n), a_data(n);
  for (size_t i = 0; i < n; ++i) {
    a_dh[i] = p;
    p += 16 + header_size(dh[i]);
  }
  for (size_t i = 0; i < n; ++i) {
    p = pad8(p);
    a_data[i] = M.sets[i].data.empty() ? kUndef : p;
    p += M.sets[i].data.size();
  }
  const uint64_t eof = pad8(p);
  // patch the placeholders
  for (size_t i = 0; i < n; ++i) {
    Out l;
    l.put(3, 1), l.put(1, 1), l.put(a_data[i], 8), l.put(M.sets[i].data.size(), 8);
    dh[i][3] = msg(0x08, 1, l.b);
  }
  {
    Out st;
    st.put(a_tree, 8), st.put(a_heap, 8);
    rh[0] = msg(0x11, 0, st.b);
  }
  // emit
  Out o;
  static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  o.bytes(sig, 8);
  o.put(0, 1), o.put(0, 1), o.put(0, 1), o.put(0, 1), o.put(0, 1), o.put(8, 1), o.put(8, 1), o.put(0, 1);
  o.put(kLeafK, 2), o.put(kNodeK, 2), o.put(0, 4);
  o.put(0, 8), o.put(kUndef, 8), o.put(eof, 8), o.put(kUndef, 8);
  o.put(0, 8), o.put(a_root, 8), o.put(1, 4), o.zeros(4), o.put(a_tree, 8), o.put(a_heap, 8);
  put_header(o, rh);
  if (o.b.size() != a_heap) fail("internal HDF5 layout error (root header)");
  o.bytes("HEAP", 4), o.put(0, 1), o.zeros(3), o.put(heapd.b.size(), 8), o.put(heap_free, 8), o.put(a_heapd, 8);
  o.bytes(heapd.b.data(), heapd.b.size());
  // group B-tree node: key 0 = "", key i+1 = the last name of node i
  std::vector<std::pair<size_t, size_t>> span(nsnod);  // [first, last) in order
  for (size_t s = 0; s < nsnod; ++s) span[s] = {s * n / nsnod, (s + 1) * n / nsnod};
  o.bytes("TREE", 4), o.put(0, 1), o.put(0, 1), o.put(n ? nsnod : 0, 2), o.put(kUndef, 8), o.put(kUndef, 8);
  const size_t tree_at = o.b.size() - 24;
  o.put(0, 8);
  for (size_t s = 0; s < nsnod && n; ++s) {
    o.put(a_snod + s * snod_size, 8);
    o.put(name_off[order[span[s].second - 1]], 8);
  }
  o.zeros(tree_at + tree_size - o.b.size());
  for (size_t s = 0; s < nsnod; ++s) {
    const size_t at = o.b.size();
    const size_t cnt = n ? span[s].second - span[s].first : 0;
    o.bytes("SNOD", 4), o.put(1, 1), o.put(0, 1), o.put(cnt, 2);
    for (size_t k = 0; k < cnt; ++k) {
      const size_t i = order[span[s].first + k];
      o.put(name_off[i], 8), o.put(a_dh[i], 8), o.put(0, 4), o.zeros(4), o.zeros(16);
    }
    o.zeros(at + snod_size - o.b.size());
  }
  for (size_t i = 0; i < n; ++i) {
    if (o.b.size() != a_dh[i]) fail("internal HDF5 layout error (dataset header)");
    put_header(o, dh[i]);
  }
  for (size_t i = 0; i < n; ++i) {
    if (M.sets[i].data.empty()) continue;
    o.align8();
    if (o.b.size() != a_data[i]) fail("internal HDF5 layout error (data)");
    o.bytes(M.sets[i].data.data(), M.sets[i].data.size());
  }
  o.align8();
  return o.b;
}

// ---------------------------------------------------------------------------------------------
// Element conversion

void swap_bytes(uint8_t *p, uint32_t size) { std::reverse(p, p + size); }

// stored elements of a scalar float/int type -> host doubles / int32
void load_f64(const Type &t, const uint8_t *src, uint64_t n, double *out) {
  for (uint64_t i = 0; i < n; ++i) {
    uint8_t e[8];
    std::memcpy(e, src + i * t.size, t.size);
    if (t.big) swap_bytes(e, t.size);
    if (t.size == 8) {
      std::memcpy(&out[i], e, 8);
    } else {
      float f;
      std::memcpy(&f, e, 4);
      out[i] = f;
    }
  }
}

void load_i32(const Type &t, const uint8_t *src, uint64_t n, int32_t *out) {
  for (uint64_t i = 0; i < n; ++i) {
    uint8_t e[8] = {0};
    std::memcpy(e, src + i * t.size, t.size);
    if (t.big) swap_bytes(e, t.size);
    int64_t v = 0;
    std::memcpy(&v, e, t.size);
    if (t.sgn && t.size < 8 && (v >> (8 * t.size - 1)) & 1) v -= (int64_t)1 << (8 * t.size);
    out[i] = (int32_t)v;
  }
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// The file handle behind kmm_io.

struct File {
  std::string path;
  bool writable = false;
  bool dirty = false;
  Model m;
};

File *create(const std::string &path, bool overwrite) {
  if (!overwrite) {
    if (FILE *f = std::fopen(path.c_str(), "rb")) {
      std::fclose(f);
      fail("create " + path + ": file exists");
    }
  }
  File *f = new File;
  f->path = path;
  f->writable = true;
  f->dirty = true;
  return f;
}

File *open(const std::string &path, bool readwrite) {
  FILE *fp = std::fopen(path.c_str(), "rb");
  if (!fp) fail("open " + path + ": cannot read the file");
  std::vector<uint8_t> bytes;
  uint8_t buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof buf, fp)) > 0) bytes.insert(bytes.end(), buf, buf + got);
  std::fclose(fp);
  std::unique_ptr<File> f(new File);
  f->path = path;
  f->writable = readwrite;
  f->m = read_model(bytes);
  return f.release();
}

void flush(File &f) {
  if (!f.writable || !f.dirty) return;
  const std::vector<uint8_t> bytes = write_model(f.m);
  const std::string tmp = f.path + ".kmm-tmp";
  FILE *fp = std::fopen(tmp.c_str(), "wb");
  if (!fp) fail("create " + f.path + ": cannot write the file");
  const bool ok = std::fwrite(bytes.data(), 1, bytes.size(), fp) == bytes.size();
  if (std::fclose(fp) != 0 || !ok || std::rename(tmp.c_str(), f.path.c_str()) != 0) {
    std::remove(tmp.c_str());
    fail("write " + f.path + ": I/O error");
  }
  f.dirty = false;
}

void string_set(File &f, const std::string &name, const std::string &value) {
  if (!f.writable) fail("attribute " + name + ": file opened read-only");
  Attr a;
  a.name = name;
  a.type = str_type((uint32_t)value.size() + 1);
  a.data.assign(value.begin(), value.end());
  a.data.push_back(0);
  auto &v = f.m.root_attrs;
  v.erase(std::remove_if(v.begin(), v.end(), [&](const Attr &x) { return x.name == name; }), v.end());
  v.push_back(a);
  f.dirty = true;
}

std::string string_get(File &f, const std::string &name) {
  for (const Attr &a : f.m.root_attrs)
    if (a.name == name) {
      if (a.type.cls != kString) fail("attribute " + name + " is not a string");
      std::string s(a.data.begin(), a.data.end());
      return s.substr(0, s.find('\0'));
    }
  fail("missing attribute " + name);
}

// What a transfer of a line, plane or field expects (module_hdf5_io.f90:212-311).
struct Want {
  std::vector<uint64_t> global;  // Fortran order: (a), (a, b) or (ny, nx/2, nz)
  int ncomp = 1;
  bool integer = false;
};

Type want_type(const Want &w) {
  Type base = w.integer ? i32() : f64();
  if (w.ncomp == 1) return base;
  Type t = f64_array((uint32_t)w.ncomp);
  return t;
}

// The checks of transfer() and legacy_layout() for an existing dataset; returns the layout.
int check_dataset(const Dataset &d, const Want &w) {
  const std::string &name = d.name;
  const int nd = (int)w.global.size();
  int layout = 0;
  if (nd == 3) {
    if (const Attr *a = d.attr("esio_field_metadata")) {
      if (a->scalar || a->dims.size() != 1) fail("malformed legacy metadata rank");
      if (a->dims[0] != 8) fail("malformed legacy metadata length");
      if (a->type.cls != kFixed) fail("malformed legacy metadata type");
      int32_t meta[8];
      load_i32(a->type, a->data.data(), 8, meta);
      layout = meta[3];
      if (layout < 0 || layout > 2) fail("unsupported legacy field layout");
      if ((uint64_t)meta[6] != w.global[0] || (uint64_t)meta[5] != w.global[1] || (uint64_t)meta[4] != w.global[2] ||
          meta[7] != w.ncomp)
        fail("legacy field metadata does not match input");
    }
  }
  const int rank = (int)d.dims.size();
  if (layout == 2) {
    if (rank != 2) fail("unexpected flattened field rank " + name);
    if (d.dims[1] != w.global[0] || d.dims[0] != w.global[1] * w.global[2])
      fail("flattened restart dimensions do not match input: " + name);
  } else {
    if (rank != nd) fail("unexpected dataset rank " + name);
    for (int i = 0; i < nd; ++i)  // C order is the Fortran order reversed
      if (d.dims[nd - 1 - i] != w.global[i]) fail("restart dimensions do not match input: " + name);
  }
  const Type *base = &d.type;
  if (w.ncomp > 1) {
    if (d.type.cls != kArray) fail("expected array-valued field " + name);
    if (d.type.adims.size() != 1) fail("unexpected component rank " + name);
    if ((int)d.type.adims[0] != w.ncomp) fail("unexpected component count " + name);
    base = d.type.base.get();
  }
  const Type e = w.integer ? i32() : f64();
  if (base->cls != e.cls || base->size != e.size) fail("unexpected numeric type " + name);
  return layout;
}

// Writes `data` (Fortran order, ncomp values per element) as dataset `name`: created if absent,
// else checked like a read and overwritten (the reference opens an existing dataset).
void write(File &f, const std::string &name, const Want &w, const void *data, const std::string &comment) {
  if (!f.writable) fail("dataset " + name + ": file opened read-only");
  uint64_t ne = 1;
  for (uint64_t g : w.global) ne *= g;
  const size_t nb = (size_t)(ne * w.ncomp * (w.integer ? 4 : 8));
  Dataset *d = f.m.find(name);
  if (!d) {
    f.m.sets.emplace_back();
    d = &f.m.sets.back();
    d->name = name;
    d->dims.assign(w.global.rbegin(), w.global.rend());
    d->type = want_type(w);
  } else {
    check_dataset(*d, w);
    // a stored byte order other than this host's is rewritten in the host's
    d->type = want_type(w);
  }
  d->data.assign(static_cast<const uint8_t *>(data), static_cast<const uint8_t *>(data) + nb);
  if (!comment.empty()) d->comment = comment;
  f.dirty = true;
}

// Reads dataset `name` into `out` (Fortran order), the elements [lo, lo + cnt) of each
// dimension (the reference's decomposition start and local sizes; an empty range reads nothing).
void read(File &f, const std::string &name, const Want &w, const std::vector<uint64_t> &lo,
          const std::vector<uint64_t> &cnt, void *out) {
  Dataset *d = f.m.find(name);
  if (!d) fail("missing restart dataset " + name);
  check_dataset(*d, w);
  const int nd = (int)w.global.size();
  uint64_t total = 1;
  for (int i = 0; i < nd; ++i) {
    if (lo[i] + cnt[i] > w.global[i]) fail("decomposition exceeds dataset");
    total *= cnt[i];
  }
  if (total == 0) return;
  const Type *base = w.ncomp > 1 ? d->type.base.get() : &d->type;
  // every layout stores the elements in the Fortran order of (global) -- walk the selection
  std::vector<uint64_t> idx(nd, 0);
  const int nc = w.ncomp;
  for (uint64_t k = 0; k < total; ++k) {
    uint64_t src = 0, stride = 1;
    for (int i = 0; i < nd; ++i) {
      src += (lo[i] + idx[i]) * stride;
      stride *= w.global[i];
    }
    const uint8_t *s = d->data.data() + src * nc * base->size;
    if (w.integer)
      load_i32(*base, s, nc, static_cast<int32_t *>(out) + k * nc);
    else
      load_f64(*base, s, nc, static_cast<double *>(out) + k * nc);
    for (int i = 0; i < nd && ++idx[i] == cnt[i]; ++i) idx[i] = 0;
  }
}

// A dataset with an explicit C-order shape and element type (tests and tools write files the
// reference's readers must refuse with these): kind 0 = float64, 1 = int32; ncomp > 1 = array.
void write_raw(File &f, const std::string &name, const std::vector<uint64_t> &cdims, int kind, int ncomp,
               const void *data) {
  if (!f.writable) fail("dataset " + name + ": file opened read-only");
  Dataset d;
  d.name = name;
  d.dims = cdims;
  d.type = kind == 1 ? i32() : f64();
  if (ncomp > 1) d.type = f64_array((uint32_t)ncomp);
  const size_t nb = (size_t)(d.elements() * d.type.size);
  d.data.assign(static_cast<const uint8_t *>(data), static_cast<const uint8_t *>(data) + nb);
  auto &v = f.m.sets;
  v.erase(std::remove_if(v.begin(), v.end(), [&](const Dataset &x) { return x.name == name; }), v.end());
  v.push_back(std::move(d));
  f.dirty = true;
}

void attr_int(File &f, const std::string &dataset, const std::string &name, int64_t n, const int32_t *v) {
  Dataset *d = f.m.find(dataset);
  if (!d) fail("missing dataset " + dataset);
  Attr a;
  a.name = name;
  a.type = i32();
  a.scalar = false;
  a.dims = {(uint64_t)n};
  a.data.assign(reinterpret_cast<const uint8_t *>(v), reinterpret_cast<const uint8_t *>(v) + 4 * n);
  auto &at = d->attrs;
  at.erase(std::remove_if(at.begin(), at.end(), [&](const Attr &x) { return x.name == name; }), at.end());
  at.push_back(a);
  f.dirty = true;
}

bool exists(File &f, const std::string &name) { return f.m.find(name) != nullptr; }

void remove(File &f, const std::string &name) {
  auto &v = f.m.sets;
  v.erase(std::remove_if(v.begin(), v.end(), [&](const Dataset &x) { return x.name == name; }), v.end());
  f.dirty = true;
}

}  // namespace h5
}  // namespace kmm

// ---------------------------------------------------------------------------------------------
// C ABI

using kmm::h5::File;
using kmm::h5::Want;

namespace {

template <typename F>
int guarded(const char *what, F &&fn) {
  try {
    fn();
    return KMM_OK;
  } catch (const std::exception &e) {
    kmm::set_error(std::string(what) + ": " + e.what());
    return KMM_ERR_IO;
  }
}

File *as_file(kmm_io *io) { return reinterpret_cast<File *>(io); }

Want line_want(int64_t n, bool integer) {
  Want w;
  w.global = {(uint64_t)n};
  w.integer = integer;
  return w;
}

}  // namespace

extern "C" {

int kmm_io_create(const char *path, int32_t overwrite, kmm_io **out) {
  if (!path || !out) return KMM_ERR_ARG;
  return guarded("kmm_io_create", [&] {
    File *f = kmm::h5::create(path, overwrite != 0);
    // io_file_create marks every file it makes (module_hdf5_io.f90:75)
    kmm::h5::string_set(*f, "Native_IO", "POONGBACK channel native parallel HDF5 v1");
    *out = reinterpret_cast<kmm_io *>(f);
  });
}

int kmm_io_open(const char *path, int32_t readwrite, kmm_io **out) {
  if (!path || !out) return KMM_ERR_ARG;
  return guarded("kmm_io_open", [&] { *out = reinterpret_cast<kmm_io *>(kmm::h5::open(path, readwrite != 0)); });
}

}  // extern "C"

namespace kmm {
void io_discard(kmm_io *io) { delete as_file(io); }
}  // namespace kmm

extern "C" {

int kmm_io_close(kmm_io *io) {
  if (!io) return KMM_ERR_ARG;
  File *f = as_file(io);
  const int rc = guarded("kmm_io_close", [&] { kmm::h5::flush(*f); });
  delete f;
  return rc;
}

int kmm_io_string_set(kmm_io *io, const char *name, const char *value) {
  if (!io || !name || !value) return KMM_ERR_ARG;
  return guarded("kmm_io_string_set", [&] { kmm::h5::string_set(*as_file(io), name, value); });
}

int kmm_io_string_get(kmm_io *io, const char *name, char *buf, int64_t len) {
  if (!io || !name || !buf || len < 1) return KMM_ERR_ARG;
  return guarded("kmm_io_string_get", [&] {
    const std::string s = kmm::h5::string_get(*as_file(io), name);
    if ((int64_t)s.size() >= len) throw kmm::h5::Error("attribute " + std::string(name) + " longer than the buffer");
    std::memcpy(buf, s.c_str(), s.size() + 1);
  });
}

int kmm_io_exists(kmm_io *io, const char *name) {
  if (!io || !name) return -KMM_ERR_ARG;
  return kmm::h5::exists(*as_file(io), name) ? 1 : 0;
}

int kmm_io_line_write_double(kmm_io *io, const char *name, int64_t n, const double *v, const char *comment) {
  if (!io || !name || !v || n < 1) return KMM_ERR_ARG;
  return guarded("kmm_io_line_write_double",
                 [&] { kmm::h5::write(*as_file(io), name, line_want(n, false), v, comment ? comment : ""); });
}

int kmm_io_line_write_integer(kmm_io *io, const char *name, int64_t n, const int32_t *v, const char *comment) {
  if (!io || !name || !v || n < 1) return KMM_ERR_ARG;
  return guarded("kmm_io_line_write_integer",
                 [&] { kmm::h5::write(*as_file(io), name, line_want(n, true), v, comment ? comment : ""); });
}

int kmm_io_line_read_double(kmm_io *io, const char *name, int64_t n, int64_t start, int64_t count, double *v) {
  if (!io || !name || n < 1 || start < 0 || count < 0 || (count > 0 && !v)) return KMM_ERR_ARG;
  return guarded("kmm_io_line_read_double", [&] {
    kmm::h5::read(*as_file(io), name, line_want(n, false), {(uint64_t)start}, {(uint64_t)count}, v);
  });
}

int kmm_io_line_read_integer(kmm_io *io, const char *name, int64_t n, int64_t start, int64_t count, int32_t *v) {
  if (!io || !name || n < 1 || start < 0 || count < 0 || (count > 0 && !v)) return KMM_ERR_ARG;
  return guarded("kmm_io_line_read_integer", [&] {
    kmm::h5::read(*as_file(io), name, line_want(n, true), {(uint64_t)start}, {(uint64_t)count}, v);
  });
}

int kmm_io_plane_write_double(kmm_io *io, const char *name, int64_t na, int64_t nb, const double *v,
                              const char *comment) {
  if (!io || !name || !v || na < 1 || nb < 1) return KMM_ERR_ARG;
  return guarded("kmm_io_plane_write_double", [&] {
    Want w;
    w.global = {(uint64_t)na, (uint64_t)nb};
    kmm::h5::write(*as_file(io), name, w, v, comment ? comment : "");
  });
}

int kmm_io_plane_read_double(kmm_io *io, const char *name, int64_t na, int64_t nb, double *v) {
  if (!io || !name || !v || na < 1 || nb < 1) return KMM_ERR_ARG;
  return guarded("kmm_io_plane_read_double", [&] {
    Want w;
    w.global = {(uint64_t)na, (uint64_t)nb};
    kmm::h5::read(*as_file(io), name, w, {0, 0}, {(uint64_t)na, (uint64_t)nb}, v);
  });
}

int kmm_io_field_writev_double(kmm_io *io, const char *name, int64_t ny, int64_t nxh, int64_t nz, int32_t ncomp,
                               const double *v) {
  if (!io || !name || !v || ny < 1 || nxh < 1 || nz < 1 || ncomp < 1) return KMM_ERR_ARG;
  return guarded("kmm_io_field_writev_double", [&] {
    Want w;
    w.global = {(uint64_t)ny, (uint64_t)nxh, (uint64_t)nz};
    w.ncomp = ncomp;
    kmm::h5::write(*as_file(io), name, w, v, "");
  });
}

int kmm_io_field_readv_double(kmm_io *io, const char *name, int64_t ny, int64_t nxh, int64_t nz, int32_t ncomp,
                              int64_t x0, int64_t xn, int64_t z0, int64_t zn, double *v) {
  if (!io || !name || ny < 1 || nxh < 1 || nz < 1 || ncomp < 1 || x0 < 0 || xn < 0 || z0 < 0 || zn < 0 ||
      (xn > 0 && zn > 0 && !v))
    return KMM_ERR_ARG;
  return guarded("kmm_io_field_readv_double", [&] {
    Want w;
    w.global = {(uint64_t)ny, (uint64_t)nxh, (uint64_t)nz};
    w.ncomp = ncomp;
    kmm::h5::read(*as_file(io), name, w, {0, (uint64_t)x0, (uint64_t)z0}, {(uint64_t)ny, (uint64_t)xn, (uint64_t)zn},
                  v);
  });
}

int kmm_io_dataset_write_raw(kmm_io *io, const char *name, int32_t rank, const int64_t *cdims, int32_t kind,
                             int32_t ncomp, const void *data) {
  if (!io || !name || rank < 0 || rank > 8 || (rank > 0 && !cdims) || !data || (kind != 0 && kind != 1) || ncomp < 1 ||
      (kind == 1 && ncomp > 1))
    return KMM_ERR_ARG;
  return guarded("kmm_io_dataset_write_raw", [&] {
    std::vector<uint64_t> d;
    for (int i = 0; i < rank; ++i) {
      if (cdims[i] < 0) throw kmm::h5::Error("negative dimension");
      d.push_back((uint64_t)cdims[i]);
    }
    kmm::h5::write_raw(*as_file(io), name, d, kind, ncomp, data);
  });
}

int kmm_io_attr_write_integer(kmm_io *io, const char *dataset, const char *name, int64_t n, const int32_t *v) {
  if (!io || !dataset || !name || n < 1 || !v) return KMM_ERR_ARG;
  return guarded("kmm_io_attr_write_integer", [&] { kmm::h5::attr_int(*as_file(io), dataset, name, n, v); });
}

int kmm_io_delete(kmm_io *io, const char *name) {
  if (!io || !name) return KMM_ERR_ARG;
  return guarded("kmm_io_delete", [&] { kmm::h5::remove(*as_file(io), name); });
}

}  // extern "C"
