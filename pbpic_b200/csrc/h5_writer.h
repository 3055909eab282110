// A minimal writer of HDF5 files (host code), enough for the reference's dump
// files: nested groups and contiguous datasets of little-endian 32/64-bit
// integers and IEEE floats, no compression, no attributes.
//
// It writes the oldest layout of the published HDF5 file format (version 0
// superblock, version 1 object headers, groups as symbol tables: a version 1
// B-tree of one leaf, a local heap of names and one symbol-table node), which
// every HDF5 library version reads:
//   superblock (96 B)              signature, sizes of offsets/lengths (8),
//                                  group K values, end of file, root entry
//   per group:  object header      one symbol-table message (B-tree, heap)
//               local heap         "HEAP" + data segment: "" at offset 0, the
//                                  children's names, a trailing free block
//               B-tree node        "TREE", type 0, one child: the SNOD
//               symbol-table node  "SNOD", entries sorted by name
//   per dataset: object header     dataspace, datatype, fill value (none
//                                  defined), contiguous layout (address, size)
//   raw data                       after all metadata, 8-byte aligned
// A group holds at most 2 * kLeafK = 256 entries (one symbol-table node).
#pragma once
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <functional>
#include <string>
#include <vector>

namespace h5w {

constexpr uint64_t kUndef = ~(uint64_t)0;
constexpr int kLeafK = 128;     // group leaf node K: 256 entries per symbol-table node
constexpr int kInternalK = 16;  // group internal node K

enum Kind { INT = 0, FLOAT = 1 };

struct Dataset {
  std::string name;
  Kind kind = FLOAT;
  int size = 4;                 // bytes per element (4 or 8)
  std::vector<uint64_t> dims;   // C order (slowest first)
  // Writes `bytes` bytes of the dataset's elements, in C order, to the file.
  std::function<bool(FILE*, uint64_t bytes)> write;
  uint64_t nbytes() const {
    uint64_t n = (uint64_t)size;
    for (uint64_t d : dims) n *= d;
    return n;
  }
};

struct Group {
  std::string name;
  std::vector<Dataset> datasets;
  std::vector<Group> groups;
};

namespace detail {

struct Buf {
  std::vector<uint8_t> b;
  void u8(uint64_t v) { b.push_back((uint8_t)v); }
  void le(uint64_t v, int n) {
    for (int i = 0; i < n; ++i) b.push_back((uint8_t)(v >> (8 * i)));
  }
  void raw(const void* p, size_t n) { b.insert(b.end(), (const uint8_t*)p, (const uint8_t*)p + n); }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  void pad8() {
    while (b.size() % 8) b.push_back(0);
  }
  void put64(size_t at, uint64_t v) {
    for (int i = 0; i < 8; ++i) b[at + i] = (uint8_t)(v >> (8 * i));
  }
};

inline size_t pad8(size_t n) { return (n + 7) & ~(size_t)7; }

// Message sizes (data part, padded to 8).
inline size_t dataspace_size(size_t rank) { return 8 + 8 * rank; }
inline size_t datatype_size(const Dataset& d) { return d.kind == INT ? 16 : 24; }
constexpr size_t kFillSize = 8;
constexpr size_t kLayoutSize = 24;
constexpr size_t kSymtabSize = 16;

inline size_t dataset_header_size(const Dataset& d) {
  return 16 + (8 + dataspace_size(d.dims.size())) + (8 + datatype_size(d)) + (8 + kFillSize) + (8 + kLayoutSize);
}
constexpr size_t kGroupHeaderSize = 16 + 8 + kSymtabSize;
constexpr size_t kHeapHeaderSize = 32;
constexpr size_t kBtreeSize = 24 + 2 * kInternalK * 8 + (2 * kInternalK + 1) * 8;
constexpr size_t kSnodSize = 8 + 2 * kLeafK * 40;

struct Entry {  // a child of a group, by name
  std::string name;
  bool group;
  uint64_t header = 0;          // object header address
  uint64_t btree = 0, heap = 0;  // groups: their symbol table
  uint64_t name_off = 0;         // offset of the name in the parent's heap
};

struct GroupLayout {
  const Group* g;
  uint64_t header, heap, heap_data, btree, snod;
  uint64_t heap_data_size, free_off;
  std::vector<Entry> entries;  // sorted by name
  std::vector<const Dataset*> dsets;  // in entry order (null for groups)
  std::vector<size_t> child_group;    // index into the layout list for group entries
};

}  // namespace detail

// Writes `root` (its name is ignored) to `path`. Returns false with a message
// in *err on failure.
inline bool write_file(const std::string& path, const Group& root, std::string* err) {
  using namespace detail;
  // ---- assign addresses: all metadata first, then the raw data
  std::vector<GroupLayout> gl;
  std::vector<std::pair<const Dataset*, uint64_t>> dheaders;  // dataset, header address
  uint64_t at = 96;
  std::function<size_t(const Group&)> place = [&](const Group& g) -> size_t {
    const size_t me = gl.size();
    gl.push_back(GroupLayout{});
    gl[me].g = &g;
    if (g.datasets.size() + g.groups.size() > (size_t)2 * kLeafK) return (size_t)-1;
    std::vector<Entry> es;
    for (const auto& c : g.groups) es.push_back(Entry{c.name, true});
    for (const auto& d : g.datasets) es.push_back(Entry{d.name, false});
    std::sort(es.begin(), es.end(), [](const Entry& a, const Entry& b) { return strcmp(a.name.c_str(), b.name.c_str()) < 0; });
    uint64_t off = 8;  // "" at offset 0
    for (auto& e : es) {
      e.name_off = off;
      off += pad8(e.name.size() + 1);
    }
    gl[me].free_off = off;
    gl[me].heap_data_size = off + 16;  // a trailing free block
    gl[me].header = at;
    at += kGroupHeaderSize;
    gl[me].heap = at;
    at += kHeapHeaderSize;
    gl[me].heap_data = at;
    at += gl[me].heap_data_size;
    gl[me].btree = at;
    at += kBtreeSize;
    gl[me].snod = at;
    at += kSnodSize;
    for (auto& e : es) {
      if (e.group) {
        const Group* c = nullptr;
        for (const auto& x : g.groups)
          if (x.name == e.name) c = &x;
        const size_t ci = place(*c);
        if (ci == (size_t)-1) return (size_t)-1;
        e.header = gl[ci].header;
        e.btree = gl[ci].btree;
        e.heap = gl[ci].heap;
        gl[me].child_group.push_back(ci);
        gl[me].dsets.push_back(nullptr);
      } else {
        const Dataset* d = nullptr;
        for (const auto& x : g.datasets)
          if (x.name == e.name) d = &x;
        e.header = at;
        at += dataset_header_size(*d);
        dheaders.push_back({d, e.header});
        gl[me].child_group.push_back((size_t)-1);
        gl[me].dsets.push_back(d);
      }
    }
    gl[me].entries = es;
    return me;
  };
  if (place(root) == (size_t)-1) {
    *err = "an HDF5 group with more than 256 entries";
    return false;
  }
  const uint64_t meta_end = at;
  std::vector<uint64_t> daddr(dheaders.size());
  at = pad8(at);
  for (size_t i = 0; i < dheaders.size(); ++i) {
    daddr[i] = at;
    at = pad8(at + dheaders[i].first->nbytes());
  }
  const uint64_t eof = at;

  // ---- metadata
  Buf m;
  // superblock
  const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  m.raw(sig, 8);
  m.u8(0); m.u8(0); m.u8(0); m.u8(0);  // superblock, free space, root entry versions, reserved
  m.u8(0); m.u8(8); m.u8(8); m.u8(0);  // shared header version, sizes of offsets and lengths, reserved
  m.le(kLeafK, 2);
  m.le(kInternalK, 2);
  m.le(0, 4);       // consistency flags
  m.le(0, 8);       // base address
  m.le(kUndef, 8);  // free space info
  m.le(eof, 8);     // end of file
  m.le(kUndef, 8);  // driver information block
  // root group symbol table entry (cache type 1: B-tree and heap in the scratch pad)
  m.le(0, 8);
  m.le(gl[0].header, 8);
  m.le(1, 4);
  m.le(0, 4);
  m.le(gl[0].btree, 8);
  m.le(gl[0].heap, 8);

  auto msg = [&](int type, size_t size, int flags) {
    m.le(type, 2);
    m.le(size, 2);
    m.u8(flags);
    m.zeros(3);
  };
  size_t di = 0;
  std::function<void(size_t)> emit = [&](size_t gi) {
    const GroupLayout& L = gl[gi];
    if (m.b.size() != L.header) return;
    // group object header: one symbol table message
    m.u8(1); m.u8(0); m.le(1, 2); m.le(1, 4); m.le(8 + kSymtabSize, 4); m.zeros(4);
    msg(0x11, kSymtabSize, 0);
    m.le(L.btree, 8);
    m.le(L.heap, 8);
    // local heap
    m.raw("HEAP", 4); m.u8(0); m.zeros(3);
    m.le(L.heap_data_size, 8);
    m.le(L.free_off, 8);
    m.le(L.heap_data, 8);
    m.zeros(8);  // ""
    for (const auto& e : L.entries) {
      m.raw(e.name.c_str(), e.name.size());
      m.zeros(pad8(e.name.size() + 1) - e.name.size());
    }
    m.le(1, 8);   // free block: next = none (1)
    m.le(16, 8);  // its size
    // B-tree: one leaf child, keys "" and the last name
    m.raw("TREE", 4); m.u8(0); m.u8(0); m.le(L.entries.empty() ? 0 : 1, 2);
    m.le(kUndef, 8); m.le(kUndef, 8);
    const size_t bt0 = m.b.size();
    m.le(0, 8);
    if (!L.entries.empty()) {
      m.le(L.snod, 8);
      m.le(L.entries.back().name_off, 8);
    }
    m.zeros(kBtreeSize - 24 - (m.b.size() - bt0));
    // symbol table node
    m.raw("SNOD", 4); m.u8(1); m.u8(0); m.le(L.entries.size(), 2);
    for (const auto& e : L.entries) {
      m.le(e.name_off, 8);
      m.le(e.header, 8);
      m.le(e.group ? 1 : 0, 4);
      m.le(0, 4);
      m.le(e.group ? e.btree : 0, 8);
      m.le(e.group ? e.heap : 0, 8);
    }
    m.zeros((size_t)(2 * kLeafK - L.entries.size()) * 40);
    // children, in entry order (addresses were assigned in this order)
    for (size_t k = 0; k < L.entries.size(); ++k) {
      if (L.entries[k].group) {
        emit(L.child_group[k]);
        continue;
      }
      const Dataset& d = *L.dsets[k];
      const size_t rank = d.dims.size();
      const size_t nmsg = 4;
      const size_t hsz = dataset_header_size(d) - 16;
      m.u8(1); m.u8(0); m.le(nmsg, 2); m.le(1, 4); m.le(hsz, 4); m.zeros(4);
      msg(0x01, dataspace_size(rank), 0);  // dataspace, version 1
      m.u8(1); m.u8((uint8_t)rank); m.u8(0); m.u8(0); m.zeros(4);
      for (uint64_t x : d.dims) m.le(x, 8);
      msg(0x03, datatype_size(d), 1);  // datatype, version 1
      if (d.kind == INT) {
        m.u8(0x10); m.u8(0x08); m.u8(0); m.u8(0);  // fixed point, little endian, signed
        m.le(d.size, 4);
        m.le(0, 2); m.le(8 * d.size, 2);
        m.zeros(4);
      } else {
        const bool dbl = d.size == 8;
        m.u8(0x11); m.u8(0x20); m.u8(dbl ? 63 : 31); m.u8(0);  // IEEE, implied msb, sign bit
        m.le(d.size, 4);
        m.le(0, 2); m.le(8 * d.size, 2);
        m.u8(dbl ? 52 : 23); m.u8(dbl ? 11 : 8); m.u8(0); m.u8(dbl ? 52 : 23);
        m.le(dbl ? 1023 : 127, 4);
        m.zeros(4);
      }
      msg(0x05, kFillSize, 1);  // fill value, version 2: allocated early, never written, undefined
      m.u8(2); m.u8(1); m.u8(2); m.u8(0); m.zeros(4);
      msg(0x08, kLayoutSize, 0);  // data layout, version 3, contiguous
      m.u8(3); m.u8(1);
      m.le(daddr[di], 8);
      m.le(d.nbytes(), 8);
      m.zeros(kLayoutSize - 18);
      ++di;
    }
  };
  emit(0);
  if (di != dheaders.size() || m.b.size() != meta_end) {
    *err = "HDF5 writer: metadata layout mismatch";
    return false;
  }
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) {
    *err = "cannot create " + path;
    return false;
  }
  bool ok = fwrite(m.b.data(), 1, m.b.size(), f) == m.b.size();
  uint64_t pos = m.b.size();
  const std::vector<uint8_t> zero(8, 0);
  for (size_t i = 0; ok && i < dheaders.size(); ++i) {
    if (pos < daddr[i]) ok = fwrite(zero.data(), 1, daddr[i] - pos, f) == daddr[i] - pos;
    pos = daddr[i];
    const uint64_t nb = dheaders[i].first->nbytes();
    if (ok && nb) ok = dheaders[i].first->write(f, nb);
    pos += nb;
  }
  if (ok && pos < eof) ok = fwrite(zero.data(), 1, eof - pos, f) == eof - pos;
  if (fclose(f) != 0) ok = false;
  if (!ok) *err = "write failed: " + path;
  return ok;
}

}  // namespace h5w
