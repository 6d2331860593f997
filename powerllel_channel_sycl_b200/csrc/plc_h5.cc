// Minimal HDF5 writer and reader (see plc_h5.h for the subset).  Layout of a
// written file: superblock (48 bytes) | root group object header | one object
// header per dataset | the raw data of each dataset (8-byte aligned).

#include "plc_h5.h"

#include <cstdio>
#include <cstring>
#include <map>

namespace plc {
namespace h5 {
namespace {

constexpr uint64_t kUndef = 0xffffffffffffffffull;
const uint8_t kSignature[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

// message types (HDF5 File Format Specification, section IV.A.2)
constexpr uint8_t kMsgDataspace = 0x01, kMsgLinkInfo = 0x02, kMsgDatatype = 0x03,
                  kMsgFillValue = 0x05, kMsgLink = 0x06, kMsgLayout = 0x08,
                  kMsgGroupInfo = 0x0A;

struct Bytes {
  std::vector<uint8_t> b;
  void u8(uint8_t x) { b.push_back(x); }
  void le(uint64_t x, int n) {
    for (int i = 0; i < n; ++i) b.push_back(uint8_t(x >> (8 * i)));
  }
  void raw(const void *p, size_t n) {
    const uint8_t *q = static_cast<const uint8_t *>(p);
    b.insert(b.end(), q, q + n);
  }
};

inline uint32_t rot(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }

size_t type_size(Type t) { return t == Type::F64 ? 8 : 4; }

uint64_t elements(const std::vector<uint64_t> &dims) {
  uint64_t n = 1;
  for (uint64_t d : dims) n *= d;
  return n;
}

// A version-2 object header holding the given messages (type, payload).
std::vector<uint8_t> object_header(const std::vector<std::pair<uint8_t, Bytes>> &msgs) {
  size_t chunk = 0;
  for (auto &m : msgs) chunk += 4 + m.second.b.size();  // type(1) size(2) flags(1) + data
  const int wflag = chunk <= 0xff ? 0 : (chunk <= 0xffff ? 1 : 2);
  const int width = 1 << wflag;
  Bytes h;
  h.raw("OHDR", 4);
  h.u8(2);      // version
  h.u8(wflag);  // flags: size-of-chunk-0 field width; no times, no attribute phase values
  h.le(chunk, width);
  for (auto &m : msgs) {
    h.u8(m.first);
    h.le(m.second.b.size(), 2);
    h.u8(0);  // message flags
    h.raw(m.second.b.data(), m.second.b.size());
  }
  h.le(lookup3(h.b.data(), h.b.size()), 4);
  return h.b;
}

std::vector<uint8_t> dataset_header(const Dataset &d, uint64_t data_addr) {
  std::vector<std::pair<uint8_t, Bytes>> msgs;
  {  // dataspace, version 2: simple, no maximum dimensions
    Bytes m;
    m.u8(2);
    m.u8(uint8_t(d.dims.size()));
    m.u8(0);
    m.u8(1);
    for (uint64_t x : d.dims) m.le(x, 8);
    msgs.push_back({kMsgDataspace, m});
  }
  {  // datatype, version 1
    Bytes m;
    if (d.type == Type::F64) {
      m.u8(0x11);  // version 1, class 1 (floating point)
      // little endian, no padding, mantissa normalisation "implied msb" (2),
      // sign bit 63
      m.u8(0x20);
      m.u8(63);
      m.u8(0);
      m.le(8, 4);
      m.le(0, 2);     // bit offset
      m.le(64, 2);    // bit precision
      m.u8(52);       // exponent location
      m.u8(11);       // exponent size
      m.u8(0);        // mantissa location
      m.u8(52);       // mantissa size
      m.le(1023, 4);  // exponent bias
    } else {
      m.u8(0x10);  // version 1, class 0 (fixed point)
      m.u8(0x08);  // little endian, signed
      m.u8(0);
      m.u8(0);
      m.le(4, 4);
      m.le(0, 2);   // bit offset
      m.le(32, 2);  // bit precision
    }
    msgs.push_back({kMsgDatatype, m});
  }
  {  // fill value, version 3: allocation early, fill written if set, none set
    Bytes m;
    m.u8(3);
    m.u8(0x01 | (0x02 << 2));
    msgs.push_back({kMsgFillValue, m});
  }
  {  // data layout, version 3: contiguous
    Bytes m;
    m.u8(3);
    m.u8(1);
    m.le(data_addr, 8);
    m.le(elements(d.dims) * type_size(d.type), 8);
    msgs.push_back({kMsgLayout, m});
  }
  return object_header(msgs);
}

std::vector<uint8_t> root_header(const std::vector<Dataset> &sets,
                                 const std::vector<uint64_t> &addrs) {
  std::vector<std::pair<uint8_t, Bytes>> msgs;
  {  // link info, version 0: no creation order, links stored in this header
    Bytes m;
    m.u8(0);
    m.u8(0);
    m.le(kUndef, 8);  // fractal heap address
    m.le(kUndef, 8);  // name index B-tree address
    msgs.push_back({kMsgLinkInfo, m});
  }
  {  // group info, version 0
    Bytes m;
    m.u8(0);
    m.u8(0);
    msgs.push_back({kMsgGroupInfo, m});
  }
  for (size_t i = 0; i < sets.size(); ++i) {  // link, version 1: hard link, 1-byte name length
    Bytes m;
    m.u8(1);
    m.u8(0);
    m.u8(uint8_t(sets[i].name.size()));
    m.raw(sets[i].name.data(), sets[i].name.size());
    m.le(addrs[i], 8);
    msgs.push_back({kMsgLink, m});
  }
  return object_header(msgs);
}

// ---- reading ----------------------------------------------------------------
// Object headers of version 1 (the library's default format) and 2, with
// their continuation blocks; groups of Link messages (compact, version-2
// superblocks) or of a symbol table (version-1 B-tree of symbol nodes over a
// local heap, version-0/1 superblocks).
struct Msg {
  uint16_t type;
  size_t at, size;
};

struct Reader {
  std::vector<uint8_t> f;
  std::string err;
  bool fail(const std::string &m) {
    err = m;
    return false;
  }
  bool have(uint64_t at, uint64_t n) const { return at <= f.size() && n <= f.size() - at; }
  uint64_t le(size_t at, int n) const {  // callers check have(at, n) first
    uint64_t x = 0;
    for (int i = 0; i < n; ++i) x |= uint64_t(f[at + i]) << (8 * i);
    return x;
  }

  // messages of a version-2 block: [at, end) holds messages with mh-byte headers
  bool v2_block(size_t at, size_t end, size_t mh, std::vector<Msg> &out,
                std::vector<std::pair<uint64_t, uint64_t>> &cont) {
    while (at + mh <= end) {
      const uint16_t type = f[at];
      const size_t size = le(at + 1, 2);
      at += mh;
      if (at + size > end) return fail("message past the object header");
      if (type == 0x10) {
        if (size < 16) return fail("bad continuation message");
        cont.emplace_back(le(at, 8), le(at + 8, 8));
      } else {
        out.push_back({type, at, size});
      }
      at += size;
    }
    return true;
  }

  bool messages(uint64_t addr, std::vector<Msg> &out) {
    std::vector<std::pair<uint64_t, uint64_t>> cont;
    if (have(addr, 16) && std::memcmp(&f[addr], "OHDR", 4) == 0) {
      if (f[addr + 4] != 2) return fail("object header version");
      const uint8_t flags = f[addr + 5];
      size_t at = addr + 6;
      if (flags & 0x20) at += 16;  // times
      if (flags & 0x10) at += 4;   // attribute phase change values
      const int width = 1 << (flags & 3);
      if (!have(at, width)) return fail("truncated object header");
      const uint64_t chunk = le(at, width);
      at += width;
      if (chunk > f.size() || !have(at, chunk + 4)) return fail("truncated object header");
      const size_t end = at + chunk;
      if (lookup3(&f[addr], end - addr) != uint32_t(le(end, 4))) return fail("object header checksum");
      const size_t mh = (flags & 0x04) ? 6 : 4;
      if (!v2_block(at, end, mh, out, cont)) return false;
      for (size_t q = 0; q < cont.size(); ++q) {  // "OCHK" blocks, checksummed
        const uint64_t b = cont[q].first, n = cont[q].second;
        if (q > 64 || n < 8 || !have(b, n) || std::memcmp(&f[b], "OCHK", 4) != 0)
          return fail("bad object header continuation block");
        if (lookup3(&f[b], n - 4) != uint32_t(le(b + n - 4, 4)))
          return fail("object header continuation checksum");
        if (!v2_block(b + 4, b + n - 4, mh, out, cont)) return false;
      }
      return true;
    }
    // version 1: version, reserved, message count (2), reference count (4),
    // header size (4), padding to 8 bytes; messages 8-byte aligned with
    // type (2), size (2), flags (1), reserved (3)
    if (!have(addr, 16) || f[addr] != 1) return fail("unknown object header");
    cont.emplace_back(addr + 16, le(addr + 8, 4));
    for (size_t q = 0; q < cont.size(); ++q) {
      const uint64_t b = cont[q].first, n = cont[q].second;
      if (q > 64 || !have(b, n)) return fail("bad object header block");
      size_t at = b;
      const size_t end = b + n;
      while (at + 8 <= end) {
        const uint16_t type = uint16_t(le(at, 2));
        const size_t size = le(at + 2, 2);
        at += 8;
        if (at + size > end) return fail("message past the object header");
        if (type == 0x10) {
          if (size < 16) return fail("bad continuation message");
          cont.emplace_back(le(at, 8), le(at + 8, 8));
        } else {
          out.push_back({type, at, size});
        }
        at += size;
      }
    }
    return true;
  }

  // members of the group whose object header is at addr: name -> header address
  bool members(uint64_t addr, std::vector<std::pair<std::string, uint64_t>> &out) {
    std::vector<Msg> msgs;
    if (!messages(addr, msgs)) return false;
    for (const Msg &m : msgs) {
      if (m.type == 0x06) {  // link
        size_t at = m.at;
        const size_t end = m.at + m.size;
        if (m.size < 2 || f[at] != 1) return fail("link message version");
        const uint8_t flags = f[at + 1];
        at += 2;
        uint8_t ltype = 0;
        if (flags & 0x08) {
          if (at >= end) return fail("bad link message");
          ltype = f[at++];
        }
        if (flags & 0x04) at += 8;
        if (flags & 0x10) at += 1;
        const int lw = 1 << (flags & 3);
        if (at + lw > end) return fail("bad link message");
        const size_t nlen = le(at, lw);
        at += lw;
        if (at + nlen > end) return fail("bad link message");
        std::string nm(reinterpret_cast<const char *>(&f[at]), nlen);
        at += nlen;
        if (ltype == 0) {
          if (at + 8 > end) return fail("bad link message");
          out.emplace_back(nm, le(at, 8));
        }
      } else if (m.type == 0x11) {  // symbol table: B-tree and local heap
        if (m.size < 16) return fail("bad symbol table message");
        if (!symbols(le(m.at, 8), le(m.at + 8, 8), out)) return false;
      }
    }
    return true;
  }

  bool symbols(uint64_t btree, uint64_t heap, std::vector<std::pair<std::string, uint64_t>> &out) {
    if (!have(heap, 32) || std::memcmp(&f[heap], "HEAP", 4) != 0) return fail("bad local heap");
    const uint64_t seg_size = le(heap + 8, 8), seg = le(heap + 24, 8);
    if (!have(seg, seg_size)) return fail("bad local heap data segment");
    std::vector<uint64_t> nodes{btree};
    for (size_t q = 0; q < nodes.size(); ++q) {
      const uint64_t n = nodes[q];
      if (q > 100000 || !have(n, 24) || std::memcmp(&f[n], "TREE", 4) != 0 || f[n + 4] != 0)
        return fail("bad group B-tree node");
      const int level = f[n + 5];
      const size_t used = le(n + 6, 2);
      // key 0 (8), child 0 (8), key 1, child 1, ..., key used
      if (!have(n + 24, 16 * used + 8)) return fail("truncated group B-tree node");
      for (size_t i = 0; i < used; ++i) {
        const uint64_t child = le(n + 24 + 8 + 16 * i, 8);
        if (level > 0) {
          nodes.push_back(child);
          continue;
        }
        if (!have(child, 8) || std::memcmp(&f[child], "SNOD", 4) != 0) return fail("bad symbol node");
        const size_t nsym = le(child + 6, 2);
        if (!have(child + 8, 40 * nsym)) return fail("truncated symbol node");
        for (size_t e = 0; e < nsym; ++e) {
          const size_t ent = child + 8 + 40 * e;
          const uint64_t name_off = le(ent, 8);
          if (name_off >= seg_size) return fail("symbol name outside the local heap");
          const char *p = reinterpret_cast<const char *>(&f[seg + name_off]);
          out.emplace_back(std::string(p, strnlen(p, seg_size - name_off)), le(ent + 8, 8));
        }
      }
    }
    return true;
  }
};

}  // namespace

uint32_t lookup3(const uint8_t *k, size_t length, uint32_t initval) {
  uint32_t a, b, c;
  a = b = c = 0xdeadbeefu + uint32_t(length) + initval;
  auto mix = [&]() {
    a -= c; a ^= rot(c, 4);  c += b;
    b -= a; b ^= rot(a, 6);  a += c;
    c -= b; c ^= rot(b, 8);  b += a;
    a -= c; a ^= rot(c, 16); c += b;
    b -= a; b ^= rot(a, 19); a += c;
    c -= b; c ^= rot(b, 4);  b += a;
  };
  while (length > 12) {
    a += k[0] + (uint32_t(k[1]) << 8) + (uint32_t(k[2]) << 16) + (uint32_t(k[3]) << 24);
    b += k[4] + (uint32_t(k[5]) << 8) + (uint32_t(k[6]) << 16) + (uint32_t(k[7]) << 24);
    c += k[8] + (uint32_t(k[9]) << 8) + (uint32_t(k[10]) << 16) + (uint32_t(k[11]) << 24);
    mix();
    length -= 12;
    k += 12;
  }
  switch (length) {  // the last block, fall through
    case 12: c += uint32_t(k[11]) << 24; [[fallthrough]];
    case 11: c += uint32_t(k[10]) << 16; [[fallthrough]];
    case 10: c += uint32_t(k[9]) << 8; [[fallthrough]];
    case 9: c += k[8]; [[fallthrough]];
    case 8: b += uint32_t(k[7]) << 24; [[fallthrough]];
    case 7: b += uint32_t(k[6]) << 16; [[fallthrough]];
    case 6: b += uint32_t(k[5]) << 8; [[fallthrough]];
    case 5: b += k[4]; [[fallthrough]];
    case 4: a += uint32_t(k[3]) << 24; [[fallthrough]];
    case 3: a += uint32_t(k[2]) << 16; [[fallthrough]];
    case 2: a += uint32_t(k[1]) << 8; [[fallthrough]];
    case 1: a += k[0]; break;
    case 0: return c;
  }
  c ^= b; c -= rot(b, 14);
  a ^= c; a -= rot(c, 11);
  b ^= a; b -= rot(a, 25);
  c ^= b; c -= rot(b, 16);
  a ^= c; a -= rot(c, 4);
  b ^= a; b -= rot(a, 14);
  c ^= b; c -= rot(b, 24);
  return c;
}

bool write_file(const std::string &path, const std::vector<Dataset> &sets, std::string &err) {
  // sizes first: the headers' lengths do not depend on the addresses
  std::vector<std::vector<uint8_t>> dh(sets.size());
  std::vector<uint64_t> hdr_addr(sets.size()), data_addr(sets.size());
  for (size_t i = 0; i < sets.size(); ++i) dh[i] = dataset_header(sets[i], 0);
  const std::vector<uint8_t> rh0 = root_header(sets, std::vector<uint64_t>(sets.size(), 0));
  uint64_t at = 48 + rh0.size();
  for (size_t i = 0; i < sets.size(); ++i) {
    hdr_addr[i] = at;
    at += dh[i].size();
  }
  for (size_t i = 0; i < sets.size(); ++i) {
    at = (at + 7) & ~uint64_t(7);
    data_addr[i] = at;
    at += elements(sets[i].dims) * type_size(sets[i].type);
  }
  const uint64_t eof = at;
  for (size_t i = 0; i < sets.size(); ++i) dh[i] = dataset_header(sets[i], data_addr[i]);
  const std::vector<uint8_t> rh = root_header(sets, hdr_addr);

  Bytes sb;  // superblock version 2
  sb.raw(kSignature, 8);
  sb.u8(2);
  sb.u8(8);  // size of offsets
  sb.u8(8);  // size of lengths
  sb.u8(0);  // consistency flags
  sb.le(0, 8);       // base address
  sb.le(kUndef, 8);  // superblock extension
  sb.le(eof, 8);
  sb.le(48, 8);      // root group object header
  sb.le(lookup3(sb.b.data(), sb.b.size()), 4);

  FILE *fp = std::fopen(path.c_str(), "wb");
  if (!fp) {
    err = "cannot create " + path;
    return false;
  }
  bool ok = std::fwrite(sb.b.data(), 1, sb.b.size(), fp) == sb.b.size() &&
            std::fwrite(rh.data(), 1, rh.size(), fp) == rh.size();
  for (size_t i = 0; ok && i < sets.size(); ++i)
    ok = std::fwrite(dh[i].data(), 1, dh[i].size(), fp) == dh[i].size();
  uint64_t pos = 48 + rh.size();
  for (auto &h : dh) pos += h.size();
  for (size_t i = 0; ok && i < sets.size(); ++i) {
    static const uint8_t zeros[8] = {0};
    if (data_addr[i] > pos) ok = std::fwrite(zeros, 1, data_addr[i] - pos, fp) == data_addr[i] - pos;
    const size_t n = elements(sets[i].dims) * type_size(sets[i].type);
    ok = ok && std::fwrite(sets[i].data, 1, n, fp) == n;
    pos = data_addr[i] + n;
  }
  ok = (std::fclose(fp) == 0) && ok;
  if (!ok) err = "write error on " + path;
  return ok;
}

bool read_dataset(const std::string &path, const std::string &name, std::vector<double> &out,
                  std::vector<uint64_t> &dims, std::string &err) {
  Reader r;
  FILE *fp = std::fopen(path.c_str(), "rb");
  if (!fp) {
    err = "PowerLLEL.ERROR.openFile: " + path + " doesn't exist!";
    return false;
  }
  std::fseek(fp, 0, SEEK_END);
  const long sz = std::ftell(fp);
  std::fseek(fp, 0, SEEK_SET);
  r.f.resize(sz > 0 ? size_t(sz) : 0);
  const bool got = std::fread(r.f.data(), 1, r.f.size(), fp) == r.f.size();
  std::fclose(fp);
  auto fail = [&](const std::string &m) {
    err = path + ": " + m;
    return false;
  };
  if (!got || r.f.size() < 48 || std::memcmp(r.f.data(), kSignature, 8) != 0)
    return fail("not an HDF5 file");
  // superblock: the root group's object header
  const uint8_t ver = r.f[8];
  uint64_t root = kUndef;
  if (ver == 2 || ver == 3) {
    if (r.f[9] != 8 || r.f[10] != 8) return fail("offset/length sizes other than 8");
    if (lookup3(r.f.data(), 44) != uint32_t(r.le(44, 4))) return fail("superblock checksum");
    root = r.le(36, 8);
  } else if (ver == 0 || ver == 1) {
    if (r.f[13] != 8 || r.f[14] != 8) return fail("offset/length sizes other than 8");
    // base, free-space, end-of-file and driver addresses, then the root
    // group's symbol table entry (link name offset, object header address)
    const size_t entry = ver == 0 ? 56 : 60;
    if (!r.have(entry, 40)) return fail("truncated superblock");
    if (r.le(entry - 32, 8) != 0) return fail("base address other than 0");
    root = r.le(entry + 8, 8);
  } else {
    return fail("superblock version " + std::to_string(ver) + " not supported");
  }
  std::vector<std::pair<std::string, uint64_t>> links;
  if (!r.members(root, links)) return fail(r.err);
  uint64_t addr = kUndef;
  for (auto &l : links)
    if (l.first == name) addr = l.second;
  if (addr == kUndef) return fail("no dataset '" + name + "' in the root group");
  std::vector<Msg> msgs;
  if (!r.messages(addr, msgs)) return fail(r.err);
  int cls = -1;
  size_t esize = 0;
  bool is_signed = true;
  uint64_t daddr = kUndef, dsize = 0;
  bool have_space = false;
  dims.clear();
  for (const Msg &m : msgs) {
    const size_t at = m.at;
    switch (m.type) {
      case kMsgDataspace: {
        if (m.size < 4) return fail("bad dataspace message");
        const int v = r.f[at], nd = r.f[at + 1];
        const size_t d0 = (v == 1) ? at + 8 : at + 4;
        if (v == 2 && r.f[at + 3] == 2) return fail("null dataspace");
        if (d0 + 8 * size_t(nd) > at + m.size) return fail("bad dataspace message");
        for (int i = 0; i < nd; ++i) dims.push_back(r.le(d0 + 8 * i, 8));
        have_space = true;
        break;
      }
      case kMsgDatatype:
        if (m.size < 8) return fail("bad datatype message");
        cls = r.f[at] & 0x0f;
        esize = r.le(at + 4, 4);
        if (r.f[at + 1] & 0x01) return fail("big-endian data not supported");
        is_signed = (r.f[at + 1] & 0x08) != 0;
        break;
      case kMsgLayout:
        if (m.size < 18 || r.f[at] != 3 || r.f[at + 1] != 1)
          return fail("only contiguous layouts are supported");
        daddr = r.le(at + 2, 8);
        dsize = r.le(at + 10, 8);
        break;
      default:
        break;
    }
  }
  if (!have_space) return fail("dataset '" + name + "' has no dataspace");
  uint64_t n = 1;
  for (uint64_t d : dims) {
    if (d != 0 && n > r.f.size() / d) return fail("dataset '" + name + "' larger than the file");
    n *= d;
  }
  if (n == 0) {
    out.clear();
    return true;
  }
  if (daddr == kUndef) return fail("dataset '" + name + "' has no data written");
  if (esize == 0 || esize > 8 || dsize != n * esize || !r.have(daddr, dsize))
    return fail("dataset '" + name + "' has no readable contiguous data");
  out.resize(n);
  const uint8_t *p = &r.f[daddr];
  for (uint64_t i = 0; i < n; ++i) {
    if (cls == 1 && esize == 8) {
      std::memcpy(&out[i], p + 8 * i, 8);
    } else if (cls == 1 && esize == 4) {
      float x;
      std::memcpy(&x, p + 4 * i, 4);
      out[i] = x;
    } else if (cls == 0 && esize == 4) {
      int32_t x;
      std::memcpy(&x, p + 4 * i, 4);
      out[i] = is_signed ? double(x) : double(uint32_t(x));
    } else if (cls == 0 && esize == 8) {
      int64_t x;
      std::memcpy(&x, p + 8 * i, 8);
      out[i] = is_signed ? double(x) : double(uint64_t(x));
    } else {
      return fail("datatype not supported");
    }
  }
  return true;
}

}  // namespace h5
}  // namespace plc
