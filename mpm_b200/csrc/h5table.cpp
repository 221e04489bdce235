// h5table.cpp -- the reference's HDF5 particle table, written and read without
// the HDF5 library.
//
// Mesh::write_particles_hdf5 (mesh.tcc:1573-1613) hands the PODParticle
// records to H5TBmake_table: one dataset named "table" in the root group, a
// one-dimensional extendible dataspace of nrecords, a compound datatype whose
// size and member offsets are the C struct's (pod_particle.cc dst_size /
// dst_offset, member types field_type: H5T_NATIVE_LLONG, _DOUBLE, _HBOOL,
// _UINT), chunked storage of 10000 records, no filters, and the table
// attributes CLASS = "TABLE", VERSION = "3.0", TITLE and FIELD_<i>_NAME.
// Mesh::read_particles_hdf5 (mesh.tcc:1663-1720) reads it back with
// H5TBread_table.  This file writes that structure with the format's original
// structures (HDF5 File Format Specification: superblock version 0, version 1
// object headers, a symbol-table root group with its local heap, version 1
// B-trees for the group and for the chunk index, datatype message version 1,
// dataspace message version 1, fill-value message version 2, layout message
// version 3, attribute messages version 1), all little-endian with 8-byte
// offsets and lengths, none of which carry checksums; and reads files of that
// structure (symbol-table groups, version 1 object headers with continuation
// blocks, compound datatypes of fixed-point and IEEE floating-point members,
// contiguous or chunked unfiltered storage).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mpm_gpu.h"

namespace {

constexpr uint64_t kUndef = ~0ull;
constexpr int kGroupLeafK = 4;       // superblock: group leaf node K
constexpr int kGroupInternalK = 16;  // superblock: group internal node K
constexpr int kChunkK = 32;          // indexed-storage B-tree K (the version 0 default)

struct Buf {
  std::vector<uint8_t> b;
  size_t size() const { return b.size(); }
  void u8(uint8_t v) { b.push_back(v); }
  void u16(uint16_t v) { put(&v, 2); }
  void u32(uint32_t v) { put(&v, 4); }
  void u64(uint64_t v) { put(&v, 8); }
  void put(const void* p, size_t n) {
    const uint8_t* c = static_cast<const uint8_t*>(p);
    b.insert(b.end(), c, c + n);
  }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  void pad8() { zeros((8 - b.size() % 8) % 8); }
  void set64(size_t at, uint64_t v) { std::memcpy(&b[at], &v, 8); }
};

// datatype message (version 1) of one member type
void put_member_type(Buf& m, int type) {
  switch (type) {
    case MPM_H5_F64:  // IEEE 754 binary64, little-endian
      m.u8(0x11);
      m.u8(0x20);  // byte order LE, no padding, mantissa normalisation: msb implied
      m.u8(63);    // sign bit position
      m.u8(0);
      m.u32(8);
      m.u16(0);   // bit offset
      m.u16(64);  // precision
      m.u8(52);   // exponent location
      m.u8(11);   // exponent size
      m.u8(0);    // mantissa location
      m.u8(52);   // mantissa size
      m.u32(1023);
      break;
    default: {  // fixed-point: size and signedness from the type code
      const bool sgn = type == MPM_H5_I64 || type == MPM_H5_I32;
      const uint32_t size = (type == MPM_H5_I64 || type == MPM_H5_U64) ? 8
                            : (type == MPM_H5_I32 || type == MPM_H5_U32) ? 4 : 1;
      m.u8(0x10);
      m.u8(sgn ? 0x08 : 0x00);  // LE, no padding, signed bit
      m.u8(0);
      m.u8(0);
      m.u32(size);
      m.u16(0);
      m.u16((uint16_t)(8 * size));
    }
  }
}

int type_size(int type) {
  switch (type) {
    case MPM_H5_F64: case MPM_H5_I64: case MPM_H5_U64: return 8;
    case MPM_H5_I32: case MPM_H5_U32: return 4;
    case MPM_H5_U8: return 1;
  }
  return -1;
}

void put_message(Buf& oh, uint16_t type, const Buf& data, uint8_t flags = 0) {
  const size_t n = (data.size() + 7) / 8 * 8;
  oh.u16(type);
  oh.u16((uint16_t)n);
  oh.u8(flags);
  oh.zeros(3);
  oh.put(data.b.data(), data.size());
  oh.zeros(n - data.size());
}

// attribute message (version 1): scalar string, null-terminated
Buf string_attribute(const std::string& name, const std::string& value) {
  Buf a;
  a.u8(1);
  a.u8(0);
  a.u16((uint16_t)(name.size() + 1));
  a.u16(8);  // datatype
  a.u16(8);  // dataspace
  a.put(name.c_str(), name.size() + 1);
  a.pad8();
  a.u8(0x13);  // string, version 1
  a.u8(0x00);  // null-terminated, ASCII
  a.u8(0);
  a.u8(0);
  a.u32((uint32_t)(value.size() + 1));
  a.u8(1);  // dataspace version 1, rank 0: scalar
  a.u8(0);
  a.u8(0);
  a.u8(0);
  a.u32(0);
  a.put(value.c_str(), value.size() + 1);
  return a;
}

}  // namespace

extern "C" int mpm_h5_write_table(const char* path, const char* title, int64_t nrecords,
                                  size_t record_size, int32_t nfields, const char* const* names,
                                  const size_t* offsets, const int32_t* types, const void* records,
                                  int64_t chunk_records) {
  if (!path || !title || nrecords < 0 || record_size == 0 || nfields <= 0 || nfields > 65535 ||
      !names || !offsets || !types || (nrecords > 0 && !records) || chunk_records <= 0)
    return MPM_ERR_INVALID;
  for (int f = 0; f < nfields; ++f) {
    const int s = type_size(types[f]);
    if (s < 0 || !names[f] || offsets[f] + (size_t)s > record_size) return MPM_ERR_INVALID;
  }
  // ---- dataset object header (its size is known before any address)
  Buf space;
  space.u8(1);
  space.u8(1);  // rank
  space.u8(1);  // maximum dimensions present
  space.u8(0);
  space.u32(0);
  space.u64((uint64_t)nrecords);
  space.u64(kUndef);  // H5S_UNLIMITED
  Buf dtype;
  dtype.u8(0x16);  // compound, version 1
  dtype.u8((uint8_t)(nfields & 0xff));
  dtype.u8((uint8_t)(nfields >> 8));
  dtype.u8(0);
  dtype.u32((uint32_t)record_size);
  for (int f = 0; f < nfields; ++f) {
    const size_t nl = std::strlen(names[f]) + 1;  // the name, null-padded to a multiple of 8
    dtype.put(names[f], nl);
    dtype.zeros((8 - nl % 8) % 8);
    dtype.u32((uint32_t)offsets[f]);
    dtype.u8(0);     // dimensionality
    dtype.zeros(3);
    dtype.u32(0);    // permutation
    dtype.u32(0);
    dtype.zeros(16); // dimension sizes
    put_member_type(dtype, types[f]);
  }
  Buf fill;
  fill.u8(2);  // version 2
  fill.u8(3);  // allocation time: incremental (chunked)
  fill.u8(2);  // write time: if set
  fill.u8(0);  // no fill value defined
  const int64_t nchunks = (nrecords + chunk_records - 1) / chunk_records;
  Buf layout;
  layout.u8(3);
  layout.u8(2);  // chunked
  layout.u8(2);  // rank + 1
  const size_t layout_addr_at = layout.size();
  layout.u64(kUndef);  // chunk B-tree address, patched below
  layout.u32((uint32_t)chunk_records);
  layout.u32((uint32_t)record_size);
  std::vector<Buf> attrs;
  attrs.push_back(string_attribute("CLASS", "TABLE"));
  attrs.push_back(string_attribute("VERSION", "3.0"));
  attrs.push_back(string_attribute("TITLE", title));
  for (int f = 0; f < nfields; ++f)
    attrs.push_back(string_attribute("FIELD_" + std::to_string(f) + "_NAME", names[f]));

  // ---- file layout: superblock, root group (header, heap, B-tree, symbol
  // node), dataset header, chunk B-tree nodes, chunks
  const uint64_t sb_size = 96;
  const uint64_t root_oh = sb_size;
  const uint64_t root_oh_size = 16 + 8 + 16;
  const uint64_t heap = root_oh + root_oh_size;
  const uint64_t heap_data = heap + 32;
  const uint64_t heap_data_size = 16;  // "" and "table"
  const uint64_t gtree = heap_data + heap_data_size;
  const uint64_t gtree_size = 24 + (2 * kGroupInternalK + 1) * 8 + 2 * kGroupInternalK * 8;
  const uint64_t snod = gtree + gtree_size;
  const uint64_t snod_size = 8 + 2 * kGroupLeafK * 40;
  const uint64_t dset_oh = snod + snod_size;
  // chunk B-tree: leaves of up to 2K chunks, parents of up to 2K children
  const uint64_t key_size = 8 + 8 * 2;
  const uint64_t node_size = 24 + (2 * kChunkK + 1) * key_size + 2 * kChunkK * 8;
  std::vector<int64_t> level_counts;  // B-tree nodes per level, leaves first; none when empty
  if (nchunks > 0) {
    int64_t n = nchunks;
    do {
      n = (n + 2 * kChunkK - 1) / (2 * kChunkK);
      level_counts.push_back(n);
    } while (n > 1);
  }
  int64_t nnodes = 0;
  for (int64_t c : level_counts) nnodes += c;
  Buf oh;  // messages of the dataset header
  put_message(oh, 0x0001, space);
  put_message(oh, 0x0003, dtype, 0x01);  // constant
  put_message(oh, 0x0005, fill, 0x01);
  const size_t layout_msg_at = oh.size() + 8;
  put_message(oh, 0x0008, layout);
  for (auto& a : attrs) put_message(oh, 0x000C, a);
  const uint64_t dset_oh_size = 16 + oh.size();
  const uint64_t tree0 = (dset_oh + dset_oh_size + 7) / 8 * 8;
  const uint64_t chunk0 = tree0 + (uint64_t)nnodes * node_size;
  const uint64_t chunk_bytes = (uint64_t)chunk_records * record_size;
  const uint64_t eof = chunk0 + (uint64_t)nchunks * chunk_bytes;

  Buf f;
  // superblock version 0
  const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  f.put(sig, 8);
  f.u8(0);  // superblock version
  f.u8(0);  // free-space version
  f.u8(0);  // root group symbol table entry version
  f.u8(0);
  f.u8(0);  // shared header message version
  f.u8(8);  // size of offsets
  f.u8(8);  // size of lengths
  f.u8(0);
  f.u16(kGroupLeafK);
  f.u16(kGroupInternalK);
  f.u32(0);  // consistency flags
  f.u64(0);  // base address
  f.u64(kUndef);
  f.u64(eof);
  f.u64(kUndef);  // driver information block
  // root group symbol table entry (cache type 1: B-tree and heap addresses)
  f.u64(0);
  f.u64(root_oh);
  f.u32(1);
  f.u32(0);
  f.u64(gtree);
  f.u64(heap);
  // root group object header: one symbol table message
  f.u8(1);
  f.u8(0);
  f.u16(1);
  f.u32(1);
  f.u32((uint32_t)(root_oh_size - 16));
  f.u32(0);
  Buf stab;
  stab.u64(gtree);
  stab.u64(heap);
  put_message(f, 0x0011, stab);
  // local heap and its data segment
  f.put("HEAP", 4);
  f.u8(0);
  f.zeros(3);
  f.u64(heap_data_size);
  f.u64(kUndef);  // no free block
  f.u64(heap_data);
  f.zeros(8);
  f.put("table\0\0\0", 8);
  // group B-tree (type 0): one child, keys "" and "table"
  {
    const size_t at = f.size();
    f.put("TREE", 4);
    f.u8(0);
    f.u8(0);
    f.u16(1);
    f.u64(kUndef);
    f.u64(kUndef);
    f.u64(0);     // key 0: ""
    f.u64(snod);  // child 0
    f.u64(8);     // key 1: "table"
    f.zeros(gtree_size - (f.size() - at));
  }
  // symbol table node
  {
    const size_t at = f.size();
    f.put("SNOD", 4);
    f.u8(1);
    f.u8(0);
    f.u16(1);
    f.u64(8);  // link name "table"
    f.u64(dset_oh);
    f.u32(0);
    f.u32(0);
    f.zeros(16);
    f.zeros(snod_size - (f.size() - at));
  }
  // dataset object header
  if (f.size() != dset_oh) return MPM_ERR_INVALID;
  {
    Buf msgs = oh;
    // the root is written last; an empty table has no chunk index
    const uint64_t tree_root = nnodes > 0 ? tree0 + (uint64_t)(nnodes - 1) * node_size : kUndef;
    std::memcpy(&msgs.b[layout_msg_at + layout_addr_at], &tree_root, 8);
    f.u8(1);
    f.u8(0);
    f.u16((uint16_t)(3 + 1 + attrs.size()));
    f.u32(1);
    f.u32((uint32_t)msgs.size());
    f.u32(0);
    f.put(msgs.b.data(), msgs.size());
  }
  f.zeros(tree0 - f.size());
  // chunk B-tree, bottom level first: node k of a level covers children
  // [k 2K, (k + 1) 2K) of the level below; keys are chunk offsets (records)
  {
    auto key = [&](Buf& b, uint32_t nbytes, uint64_t offset) {
      b.u32(nbytes);
      b.u32(0);  // filter mask
      b.u64(offset);
      b.u64(0);
    };
    int64_t below = nchunks;  // children of the current level
    uint64_t below_addr = chunk0;                   // address of child 0 of the level below
    uint64_t below_stride = chunk_bytes;
    uint64_t span = (uint64_t)chunk_records;  // records under one child
    uint64_t addr = tree0;
    for (size_t lv = 0; lv < level_counts.size(); ++lv) {
      const int64_t nodes = level_counts[lv];
      for (int64_t k = 0; k < nodes; ++k) {
        const size_t at = f.size();
        const int64_t c0 = k * 2 * kChunkK;
        const int64_t c1 = std::min<int64_t>(below, c0 + 2 * kChunkK);
        f.put("TREE", 4);
        f.u8(1);
        f.u8((uint8_t)lv);
        f.u16((uint16_t)(c1 - c0));
        f.u64(k > 0 ? addr - node_size : kUndef);
        f.u64(k + 1 < nodes ? addr + node_size : kUndef);
        for (int64_t c = c0; c < c1; ++c) {
          key(f, lv == 0 ? (uint32_t)chunk_bytes : 0, (uint64_t)c * span);
          f.u64(below_addr + (uint64_t)c * below_stride);
        }
        key(f, 0, (uint64_t)c1 * span);
        f.zeros(node_size - (f.size() - at));
        addr += node_size;
      }
      below_addr = addr - (uint64_t)nodes * node_size;
      below_stride = node_size;
      below = nodes;
      span *= 2 * kChunkK;
    }
  }
  if (f.size() != chunk0) return MPM_ERR_INVALID;
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return MPM_ERR_INVALID;
  bool ok = std::fwrite(f.b.data(), 1, f.size(), fp) == f.size();
  const uint8_t* rec = static_cast<const uint8_t*>(records);
  for (int64_t c = 0; c < nchunks && ok; ++c) {
    const int64_t r0 = c * chunk_records, r1 = std::min<int64_t>(nrecords, r0 + chunk_records);
    ok = std::fwrite(rec + (size_t)r0 * record_size, record_size, (size_t)(r1 - r0), fp) ==
         (size_t)(r1 - r0);
    if (ok && r1 - r0 < chunk_records) {  // the last chunk is stored whole
      std::vector<uint8_t> z((size_t)(chunk_records - (r1 - r0)) * record_size, 0);
      ok = std::fwrite(z.data(), 1, z.size(), fp) == z.size();
    }
  }
  ok = std::fclose(fp) == 0 && ok;
  return ok ? MPM_OK : MPM_ERR_INVALID;
}

// ------------------------------------------------------------------ reader
namespace {

struct File {
  std::vector<uint8_t> d;
  uint64_t u(uint64_t at, int n) const {
    if (at + n > d.size()) throw std::runtime_error("HDF5 file truncated");
    uint64_t v = 0;
    std::memcpy(&v, &d[at], n);
    return v;
  }
  std::string str(uint64_t at) const {
    std::string s;
    while (at < d.size() && d[at]) s += (char)d[at++];
    return s;
  }
};

struct Member {
  std::string name;
  uint64_t offset;
  int type;  // MPM_H5_*
};

struct Table {
  uint64_t nrecords = 0, record_size = 0;
  std::vector<Member> members;
  int layout = -1;  // 1 contiguous, 2 chunked
  uint64_t data_addr = kUndef, chunk_records = 0;
};

int decode_type(const File& f, uint64_t at, uint64_t* size_out, uint64_t* len) {
  const int cls = f.u(at, 1) & 0x0f;
  const uint64_t bits = f.u(at + 1, 3);
  const uint64_t size = f.u(at + 4, 4);
  *size_out = size;
  if (cls == 0) {  // fixed-point
    if (bits & 1) throw std::runtime_error("big-endian member");
    *len = 12;
    const bool sgn = (bits >> 3) & 1;
    if (size == 8) return sgn ? MPM_H5_I64 : MPM_H5_U64;
    if (size == 4) return sgn ? MPM_H5_I32 : MPM_H5_U32;
    if (size == 1) return MPM_H5_U8;
    throw std::runtime_error("unsupported integer size");
  }
  if (cls == 1) {
    if ((bits & 1) || size != 8) throw std::runtime_error("unsupported floating-point member");
    *len = 20;
    return MPM_H5_F64;
  }
  throw std::runtime_error("unsupported member class " + std::to_string(cls));
}

void parse_messages(const File& f, uint64_t at, uint64_t size, Table& t) {
  const uint64_t end = at + size;
  while (at + 8 <= end) {
    const uint64_t type = f.u(at, 2), msize = f.u(at + 2, 2);
    const uint64_t m = at + 8;
    if (type == 0x0001) {  // dataspace
      const int ver = (int)f.u(m, 1), rank = (int)f.u(m + 1, 1);
      if (rank != 1) throw std::runtime_error("table dataspace is not one-dimensional");
      t.nrecords = f.u(m + (ver == 1 ? 8 : 4), 8);
    } else if (type == 0x0003) {  // datatype
      const int cls = f.u(m, 1) & 0x0f, ver = (int)(f.u(m, 1) >> 4);
      if (cls != 6) throw std::runtime_error("table datatype is not compound");
      const uint64_t nm = f.u(m + 1, 2);
      t.record_size = f.u(m + 4, 4);
      uint64_t p = m + 8;
      for (uint64_t i = 0; i < nm; ++i) {
        Member mb;
        mb.name = f.str(p);
        if (ver >= 3) {
          p += mb.name.size() + 1;
          int nb = 1;
          while ((t.record_size >> (8 * nb)) && nb < 8) ++nb;
          mb.offset = f.u(p, nb);
          p += nb;
        } else {
          p += (mb.name.size() + 1 + 7) / 8 * 8;
          mb.offset = f.u(p, 4);
          p += ver == 1 ? 32 : 4;
        }
        uint64_t sz = 0, len = 0;
        mb.type = decode_type(f, p, &sz, &len);
        p += len;
        t.members.push_back(mb);
      }
    } else if (type == 0x0008) {  // layout
      if (f.u(m, 1) != 3) throw std::runtime_error("unsupported layout message version");
      t.layout = (int)f.u(m + 1, 1);
      if (t.layout == 1) {
        t.data_addr = f.u(m + 2, 8);
      } else if (t.layout == 2) {
        t.data_addr = f.u(m + 3, 8);
        t.chunk_records = f.u(m + 11, 4);
      } else {
        throw std::runtime_error("compact table storage is not read");
      }
    } else if (type == 0x000B) {
      throw std::runtime_error("filtered (compressed) table storage is not read");
    } else if (type == 0x0010) {  // continuation
      parse_messages(f, f.u(m, 8), f.u(m + 8, 8), t);
    }
    at = m + msize;
  }
}

// chunk index: (offset in records, address) of every chunk, in order
void collect_chunks(const File& f, uint64_t node, std::vector<std::pair<uint64_t, uint64_t>>& out) {
  if (f.u(node, 4) != 0x45455254u) throw std::runtime_error("bad chunk B-tree node");  // "TREE"
  if (f.u(node + 4, 1) != 1) throw std::runtime_error("not a chunk B-tree");
  const int level = (int)f.u(node + 5, 1);
  const uint64_t n = f.u(node + 6, 2);
  const uint64_t ks = 8 + 8 * 2;
  uint64_t p = node + 24;
  for (uint64_t i = 0; i < n; ++i) {
    if (f.u(p + 4, 4) != 0) throw std::runtime_error("filtered chunk");
    const uint64_t off = f.u(p + 8, 8);
    const uint64_t child = f.u(p + ks, 8);
    if (level == 0)
      out.emplace_back(off, child);
    else
      collect_chunks(f, child, out);
    p += ks + 8;
  }
}

uint64_t find_table(const File& f) {
  if (f.u(0, 4) != 0x46444889u) throw std::runtime_error("not an HDF5 file");
  if (f.u(8, 1) != 0 && f.u(8, 1) != 1) throw std::runtime_error("unsupported superblock version");
  if (f.u(13, 1) != 8 || f.u(14, 1) != 8) throw std::runtime_error("offsets and lengths must be 8 bytes");
  const uint64_t entry = f.u(8, 1) == 0 ? 56 : 64;
  const uint64_t root_oh = f.u(entry + 8, 8);
  // the root header's symbol table message
  uint64_t btree = kUndef, heap = kUndef;
  if (f.u(root_oh, 1) != 1) throw std::runtime_error("unsupported root object header");
  const uint64_t nmsg = f.u(root_oh + 2, 2);
  uint64_t at = root_oh + 16;
  for (uint64_t i = 0; i < nmsg; ++i) {
    const uint64_t type = f.u(at, 2), ms = f.u(at + 2, 2);
    if (type == 0x0011) {
      btree = f.u(at + 8, 8);
      heap = f.u(at + 16, 8);
    }
    at += 8 + ms;
  }
  if (btree == kUndef) throw std::runtime_error("root group is not a symbol-table group");
  const uint64_t heap_data = f.u(heap + 24, 8);
  std::vector<uint64_t> stack{btree};
  while (!stack.empty()) {
    const uint64_t node = stack.back();
    stack.pop_back();
    const int level = (int)f.u(node + 5, 1);
    const uint64_t n = f.u(node + 6, 2);
    for (uint64_t i = 0; i < n; ++i) {
      const uint64_t child = f.u(node + 24 + 8 + i * 16, 8);
      if (level > 0) {
        stack.push_back(child);
        continue;
      }
      const uint64_t ns = f.u(child + 6, 2);
      for (uint64_t k = 0; k < ns; ++k) {
        const uint64_t e = child + 8 + k * 40;
        if (f.str(heap_data + f.u(e, 8)) == "table") return f.u(e + 8, 8);
      }
    }
  }
  throw std::runtime_error("no dataset named \"table\"");
}

Table read_table(const File& f) {
  const uint64_t oh = find_table(f);
  if (f.u(oh, 1) != 1) throw std::runtime_error("unsupported dataset object header");
  Table t;
  parse_messages(f, oh + 16, f.u(oh + 8, 4), t);
  if (t.layout < 0 || t.members.empty()) throw std::runtime_error("incomplete table dataset");
  return t;
}

}  // namespace

extern "C" int mpm_h5_read_table(const char* path, int64_t* nrecords, size_t record_size,
                                 int32_t nfields, const char* const* names, const size_t* offsets,
                                 const int32_t* types, void* records, int64_t capacity, char* err,
                                 int64_t errlen) {
  auto fail = [&](const std::string& m) {
    if (err && errlen > 0) std::snprintf(err, (size_t)errlen, "%s", m.c_str());
    return MPM_ERR_INVALID;
  };
  if (!path || !nrecords) return fail("null argument");
  try {
    File f;
    {
      FILE* fp = std::fopen(path, "rb");
      if (!fp) return fail(std::string("cannot open ") + path);
      std::fseek(fp, 0, SEEK_END);
      const long n = std::ftell(fp);
      std::fseek(fp, 0, SEEK_SET);
      f.d.resize(n > 0 ? (size_t)n : 0);
      const size_t got = n > 0 ? std::fread(f.d.data(), 1, (size_t)n, fp) : 0;
      std::fclose(fp);
      if (got != f.d.size()) return fail("cannot read the file");
    }
    const Table t = read_table(f);
    *nrecords = (int64_t)t.nrecords;
    if (!records) return MPM_OK;  // size query
    if ((int64_t)t.nrecords > capacity) return fail("capacity below the table's record count");
    // field map: the caller's fields by name
    std::vector<const Member*> src(nfields, nullptr);
    for (int k = 0; k < nfields; ++k) {
      for (const Member& m : t.members)
        if (m.name == names[k]) src[k] = &m;
      if (!src[k]) return fail(std::string("table has no field ") + names[k]);
      if (src[k]->type != types[k]) return fail(std::string("field ") + names[k] + " has another type");
    }
    std::vector<std::pair<uint64_t, uint64_t>> chunks;  // (first record, address)
    if (t.layout == 1)
      chunks.emplace_back(0, t.data_addr);
    else if (t.nrecords > 0 && t.data_addr != kUndef)
      collect_chunks(f, t.data_addr, chunks);
    uint8_t* out = static_cast<uint8_t*>(records);
    const uint64_t span = t.layout == 1 ? t.nrecords : t.chunk_records;
    for (const auto& ch : chunks) {
      for (uint64_t r = 0; r < span && ch.first + r < t.nrecords; ++r) {
        const uint64_t at = ch.second + r * t.record_size;
        uint8_t* dst = out + (size_t)(ch.first + r) * record_size;
        for (int k = 0; k < nfields; ++k) {
          const int s = type_size(types[k]);
          if (at + src[k]->offset + s > f.d.size()) return fail("record beyond the end of the file");
          std::memcpy(dst + offsets[k], &f.d[at + src[k]->offset], (size_t)s);
        }
      }
    }
  } catch (const std::exception& e) {
    return fail(e.what());
  }
  return MPM_OK;
}
