// h5beam.cpp -- Bmad's openPMD beam file in HDF5, read and written without the HDF5 library.
//
// The layout is the reference's: hdf5_write_beam (bmad/hdf5/hdf5_write_beam.f90:20-245) writes one
// group per bunch under basePath "/data/%T/" ("/data/00001/", ...), a "particles/" group with one
// species group inside it (the old layout puts the records in "particles/" directly), and one
// record per quantity: a dataset of n values when they differ, else a "constant record component"
// (pmd_write_real_to_pseudo_dataset, hdf5_openpmd_mod.f90:515-537: a group with attributes value
// and shape). Every record carries localName, unitSI, unitDimension and unitSymbol.
// hdf5_read_beam (bmad/hdf5/hdf5_read_beam.f90:24-474, called without an element) rebuilds the
// coordinates: pz from totalMomentum / p0c, px and py from momentum / p0c, beta from (1 + pz) p0c
// and the mass, z = -beta c dt, t = timeOffset + time, and the location from -1/0/1.
//
// The image has no HDF5 library, so the file format is handled here. Both sides use the classic
// structures that libhdf5 writes by default (the reference's own test file bunch_old.h5 is built of
// them): superblock version 0, version-1 object headers (with continuation blocks on reading),
// groups as symbol tables (a version-1 B-tree of symbol-table nodes, names in a local heap),
// contiguous or compact dataset storage, version-1 attribute messages, little-endian integers and
// IEEE doubles, fixed-length strings. Files that use the newer structures (superblock 2/3, version-2
// object headers, link messages, chunked or filtered storage) are refused with BMADGPU_EUNSUPPORTED.
// The particle species comes from the caller's bmadgpu_param, as for the ASCII reader; photon
// bunches (speciesType "photon") are refused.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "../../include/bmadgpu.h"

namespace {

constexpr uint64_t kUndef = ~0ull;
constexpr double kCLight = 2.99792458e8;         // physical_constants.f90
constexpr double kECharge = 1.602176634e-19;
constexpr double kHbar = 4.135667696e-15 / (2 * 3.141592653589793238462643383279502884197);   // [eV s]

// ---- reading ---------------------------------------------------------------------------------

struct Err {
  int code;
};

struct Type {
  int cls = -1;  // 0 fixed-point, 1 float, 3 string
  int size = 0;
  bool is_signed = true;
};

struct Attr {
  Type type;
  uint64_t count = 0;
  const uint8_t* data = nullptr;
};

struct Object {
  bool is_group = false, is_dataset = false;
  uint64_t btree = 0, heap = 0;                       // symbol table
  Type type;                                           // dataset
  uint64_t count = 0;
  const uint8_t* data = nullptr;                       // compact or contiguous data (nullptr: unallocated)
  uint64_t data_bytes = 0;
  std::map<std::string, Attr> attrs;
  struct Raw {
    int type, flags;
    const uint8_t* body;
    uint64_t size;
  };
  std::vector<Raw> raw;                                // every message, for copying the object
};

class Reader {
 public:
  explicit Reader(std::vector<uint8_t> bytes) : d_(std::move(bytes)) {}

  uint64_t u(uint64_t off, int n) const {
    if (off + n > d_.size()) throw Err{BMADGPU_EINVAL};
    uint64_t v = 0;
    for (int i = n - 1; i >= 0; i--) v = (v << 8) | d_[off + i];
    return v;
  }
  const uint8_t* at(uint64_t off, uint64_t n) const {
    if (off > d_.size() || n > d_.size() - off) throw Err{BMADGPU_EINVAL};
    return d_.data() + off;
  }

  // Superblock: signature at 0, 512, 1024, ...; version 0 or 1 with 8-byte offsets and lengths.
  uint64_t root() {
    static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    for (uint64_t sb = 0; sb + 96 <= d_.size(); sb = sb ? sb * 2 : 512) {
      if (std::memcmp(d_.data() + sb, sig, 8) != 0) continue;
      const int ver = d_[sb + 8];
      if (ver > 1 || d_[sb + 13] != 8 || d_[sb + 14] != 8) throw Err{BMADGPU_EUNSUPPORTED};
      base_ = u(sb + 24 + (ver == 1 ? 4 : 0), 8);
      return u(sb + (ver == 1 ? 60 : 56) + 8, 8);     // root symbol-table entry: object header address
    }
    throw Err{BMADGPU_EINVAL};
  }

  static Type parse_type(const uint8_t* p) {
    Type t;
    t.cls = p[0] & 15;
    t.size = (int)(p[4] | p[5] << 8 | p[6] << 16 | (uint32_t)p[7] << 24);
    if (t.cls == 0) {
      if (p[1] & 1) throw Err{BMADGPU_EUNSUPPORTED};   // big-endian
      t.is_signed = (p[1] & 8) != 0;
      if (t.size != 1 && t.size != 2 && t.size != 4 && t.size != 8) throw Err{BMADGPU_EUNSUPPORTED};
    } else if (t.cls == 1) {
      if ((p[1] & 1) || (t.size != 4 && t.size != 8)) throw Err{BMADGPU_EUNSUPPORTED};
    } else if (t.cls != 3) {
      throw Err{BMADGPU_EUNSUPPORTED};
    }
    return t;
  }

  // Dataspace message (versions 1 and 2) of len bytes: number of elements.
  static uint64_t parse_space(const uint8_t* p, uint64_t len) {
    if (len < 4) throw Err{BMADGPU_EINVAL};
    const int ver = p[0], rank = p[1];
    if (ver != 1 && ver != 2) throw Err{BMADGPU_EUNSUPPORTED};
    if (ver == 2 && p[3] == 2) return 0;               // null dataspace
    const uint64_t head = ver == 1 ? 8 : 4;
    if (head + 8 * (uint64_t)rank > len) throw Err{BMADGPU_EINVAL};
    const uint8_t* dims = p + head;
    uint64_t n = 1;
    for (int i = 0; i < rank; i++) {
      uint64_t v = 0;
      for (int b = 7; b >= 0; b--) v = (v << 8) | dims[8 * i + b];
      if (__builtin_mul_overflow(n, v, &n)) throw Err{BMADGPU_EINVAL};
    }
    return n;
  }

  Object object(uint64_t addr) {
    addr += base_;
    if (u(addr, 1) != 1) throw Err{BMADGPU_EUNSUPPORTED};   // "OHDR": version-2 object header
    const uint64_t n_msgs = u(addr + 2, 2);
    std::vector<std::pair<uint64_t, uint64_t>> blocks{{addr + 16, u(addr + 8, 4)}};
    Object o;
    uint64_t seen = 0;
    for (size_t bi = 0; bi < blocks.size() && seen < n_msgs; bi++) {
      uint64_t p = blocks[bi].first;
      const uint64_t end = p + blocks[bi].second;
      while (p + 8 <= end && seen < n_msgs) {
        const int type = (int)u(p, 2);
        const uint64_t size = u(p + 2, 2);
        const uint64_t body = p + 8;
        const uint8_t* b = at(body, size);
        seen++;
        o.raw.push_back({type, (int)u(p + 4, 1), b, size});
        switch (type) {
          case 0x01: o.count = parse_space(b, size); break;
          case 0x03:
            if (size < 8) throw Err{BMADGPU_EINVAL};
            o.type = parse_type(b);
            break;
          case 0x08: {
            if (size < 4) throw Err{BMADGPU_EINVAL};
            if (b[0] != 3) throw Err{BMADGPU_EUNSUPPORTED};
            o.is_dataset = true;
            if (b[1] == 0) {
              o.data_bytes = u(body + 2, 2);               // compact: size (2), raw data
              o.data = at(body + 4, o.data_bytes);
            } else if (b[1] == 1) {
              const uint64_t a = u(body + 2, 8);
              o.data_bytes = u(body + 10, 8);
              o.data = a == kUndef ? nullptr : at(a + base_, o.data_bytes);
            } else {
              throw Err{BMADGPU_EUNSUPPORTED};             // chunked or virtual storage
            }
            break;
          }
          case 0x0B: throw Err{BMADGPU_EUNSUPPORTED};      // filter pipeline
          case 0x0C: parse_attr(b, size, o); break;
          case 0x10: blocks.push_back({u(body, 8) + base_, u(body + 8, 8)}); break;
          case 0x11: o.is_group = true; o.btree = u(body, 8); o.heap = u(body + 8, 8); break;
          case 0x06: case 0x02: throw Err{BMADGPU_EUNSUPPORTED};   // link messages (new-style groups)
          default: break;
        }
        p = body + size;
      }
    }
    return o;
  }

  // Attribute message, versions 1 (fields padded to 8 bytes), 2 and 3.
  void parse_attr(const uint8_t* b, uint64_t size, Object& o) {
    const int ver = b[0];
    if (ver < 1 || ver > 3) throw Err{BMADGPU_EUNSUPPORTED};
    const int nl = b[2] | b[3] << 8, tl = b[4] | b[5] << 8, sl = b[6] | b[7] << 8;
    auto pad = [&](int x) { return ver == 1 ? (x + 7) / 8 * 8 : x; };
    if (8u + (ver == 3 ? 1 : 0) + pad(nl) + pad(tl) + pad(sl) > size || tl < 8 || sl < 4) throw Err{BMADGPU_EINVAL};
    const uint8_t* q = b + 8 + (ver == 3 ? 1 : 0);
    std::string name((const char*)q, strnlen((const char*)q, nl));
    q += pad(nl);
    Attr a;
    a.type = parse_type(q);
    q += pad(tl);
    a.count = parse_space(q, sl);
    q += pad(sl);
    a.data = q;
    uint64_t bytes;
    if (q > b + size || __builtin_mul_overflow(a.count, (uint64_t)a.type.size, &bytes) ||
        bytes > (uint64_t)(b + size - q))
      throw Err{BMADGPU_EINVAL};
    if (a.count > 0) o.attrs[name] = a;                // an attribute without a value reads as absent
  }

  std::string heap_name(uint64_t heap, uint64_t off) {
    heap += base_;
    if (std::memcmp(at(heap, 4), "HEAP", 4) != 0) throw Err{BMADGPU_EINVAL};
    const uint64_t seg = u(heap + 24, 8) + base_, size = u(heap + 8, 8);
    const char* s = (const char*)at(seg, size);
    if (off >= size) throw Err{BMADGPU_EINVAL};
    return std::string(s + off, strnlen(s + off, size - off));
  }

  // Children of a symbol-table group: (name, object header address), in the B-tree's name order.
  void children(uint64_t btree, uint64_t heap, std::vector<std::pair<std::string, uint64_t>>& out, int depth = 0) {
    if (depth > 32) throw Err{BMADGPU_EINVAL};
    const uint64_t t = btree + base_;
    if (std::memcmp(at(t, 4), "TREE", 4) != 0 || u(t + 4, 1) != 0) throw Err{BMADGPU_EINVAL};
    const int level = (int)u(t + 5, 1), used = (int)u(t + 6, 2);
    for (int i = 0; i < used; i++) {
      const uint64_t child = u(t + 24 + 8 + 16 * (uint64_t)i, 8);
      if (level > 0) { children(child, heap, out, depth + 1); continue; }
      const uint64_t s = child + base_;
      if (std::memcmp(at(s, 4), "SNOD", 4) != 0) throw Err{BMADGPU_EINVAL};
      const int n = (int)u(s + 6, 2);
      for (int j = 0; j < n; j++) {
        const uint64_t e = s + 8 + 40 * (uint64_t)j;
        out.push_back({heap_name(heap, u(e, 8)), u(e + 8, 8)});
      }
    }
  }

  // Object at a slash-separated path below a group's object header address.
  bool lookup(uint64_t from, const std::string& path, uint64_t* addr) {
    uint64_t cur = from;
    size_t i = 0;
    while (i < path.size()) {
      size_t j = path.find('/', i);
      if (j == std::string::npos) j = path.size();
      const std::string part = path.substr(i, j - i);
      i = j + 1;
      if (part.empty() || part == ".") continue;
      Object g = object(cur);
      if (!g.is_group) return false;
      std::vector<std::pair<std::string, uint64_t>> ch;
      children(g.btree, g.heap, ch);
      bool found = false;
      for (auto& c : ch)
        if (c.first == part) { cur = c.second; found = true; break; }
      if (!found) return false;
    }
    *addr = cur;
    return true;
  }

  static double real_at(const Type& t, const uint8_t* p) {
    if (t.cls == 1) {
      if (t.size == 8) { double v; std::memcpy(&v, p, 8); return v; }
      float v; std::memcpy(&v, p, 4); return v;
    }
    if (t.cls == 0) return (double)int_at(t, p);
    throw Err{BMADGPU_EINVAL};
  }
  static int64_t int_at(const Type& t, const uint8_t* p) {
    if (t.cls == 1) return (int64_t)real_at(t, p);
    if (t.cls != 0) throw Err{BMADGPU_EINVAL};
    uint64_t v = 0;
    for (int b = t.size - 1; b >= 0; b--) v = (v << 8) | p[b];
    if (t.is_signed && t.size < 8 && (v >> (8 * t.size - 1)) & 1) v |= ~0ull << (8 * t.size);
    return (int64_t)v;
  }
  static std::string str(const Attr& a) {
    if (a.type.cls != 3) throw Err{BMADGPU_EINVAL};
    const char* s = (const char*)a.data;
    std::string v(s, strnlen(s, a.type.size));
    while (!v.empty() && v.back() == ' ') v.pop_back();   // space-padded strings
    return v;
  }

 private:
  std::vector<uint8_t> d_;
  uint64_t base_ = 0;
};

// One openPMD record (dataset, or constant record component) of n values, scaled as
// pmd_read_real_dataset_rank1 does (hdf5_openpmd_mod.f90:1050-1099): array * (factor / unitSI)
// unless unitSI equals the factor to 1e-15.
bool read_record(Reader& r, uint64_t species, const std::string& name, double factor, int64_t n,
                 std::vector<double>& out) {
  uint64_t addr;
  if (!r.lookup(species, name, &addr)) return false;
  Object o = r.object(addr);
  auto it = o.attrs.find("unitSI");
  if (it == o.attrs.end() || it->second.count < 1) throw Err{BMADGPU_EINVAL};
  const double unit_si = Reader::real_at(it->second.type, it->second.data);
  out.assign(n, 0.0);
  if (o.is_dataset) {
    if ((int64_t)o.count != n) throw Err{BMADGPU_EINVAL};
    uint64_t need;
    if (__builtin_mul_overflow((uint64_t)n, (uint64_t)o.type.size, &need) || (o.data && o.data_bytes < need))
      throw Err{BMADGPU_EINVAL};
    if (o.data)
      for (int64_t j = 0; j < n; j++) out[j] = Reader::real_at(o.type, o.data + (uint64_t)j * o.type.size);
  } else {
    auto v = o.attrs.find("value");
    if (v == o.attrs.end()) throw Err{BMADGPU_EINVAL};
    const double c = Reader::real_at(v->second.type, v->second.data);
    for (auto& x : out) x = c;
  }
  if (std::fabs(unit_si - factor) > 1e-15 * factor)
    for (auto& x : out) x *= factor / unit_si;
  return true;
}

bool read_int_record(Reader& r, uint64_t species, const std::string& name, int64_t n, std::vector<int64_t>& out) {
  uint64_t addr;
  if (!r.lookup(species, name, &addr)) return false;
  Object o = r.object(addr);
  out.assign(n, 0);
  if (o.is_dataset) {
    if ((int64_t)o.count != n) throw Err{BMADGPU_EINVAL};
    uint64_t need;
    if (__builtin_mul_overflow((uint64_t)n, (uint64_t)o.type.size, &need) || (o.data && o.data_bytes < need))
      throw Err{BMADGPU_EINVAL};
    if (o.data)
      for (int64_t j = 0; j < n; j++) out[j] = Reader::int_at(o.type, o.data + (uint64_t)j * o.type.size);
  } else {
    auto v = o.attrs.find("value");
    if (v == o.attrs.end()) throw Err{BMADGPU_EINVAL};
    const int64_t c = Reader::int_at(v->second.type, v->second.data);
    for (auto& x : out) x = c;
  }
  return true;
}

bool is_integer(const std::string& s) {
  if (s.empty()) return false;
  for (char c : s)
    if (c < '0' || c > '9') return false;
  return true;
}

int read_hdf5(const char* path, const bmadgpu_param* param, int32_t ix_bunch, int32_t flags, bmadgpu_bunch* b,
              int64_t* n_particle, int32_t* n_bunch) {
  const bool at_ele = (flags & BMADGPU_BEAM_AT_ELEMENT) != 0;
  FILE* f = std::fopen(path, "rb");
  if (!f) return BMADGPU_EINVAL;
  std::vector<uint8_t> bytes;
  uint8_t buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) bytes.insert(bytes.end(), buf, buf + got);
  std::fclose(f);
  Reader r(std::move(bytes));
  const uint64_t root = r.root();
  Object ro = r.object(root);
  auto attr_str = [&](const char* k) -> std::string {
    auto it = ro.attrs.find(k);
    if (it == ro.attrs.end()) throw Err{BMADGPU_EINVAL};
    return Reader::str(it->second);
  };
  const std::string base_path = attr_str("basePath"), particles_path = attr_str("particlesPath");
  std::string software;
  if (ro.attrs.count("software")) software = Reader::str(ro.attrs["software"]);

  // The bunch groups: basePath without "%T" names the one bunch; with it, every group of the
  // directory before "%T" whose name matches around an integer (hdf5_read_beam.f90:100-160).
  std::vector<std::string> bunch_paths;
  const size_t it_t = base_path.find("%T");
  if (it_t == std::string::npos) {
    bunch_paths.push_back(base_path);
  } else {
    const size_t is = base_path.rfind('/', it_t);
    const std::string dir = base_path.substr(0, is == std::string::npos ? 0 : is + 1);
    std::string t_match = base_path.substr(is == std::string::npos ? 0 : is + 1);
    if (!t_match.empty() && t_match.back() == '/') t_match.pop_back();
    std::string sub_dir;
    const size_t slash = t_match.find('/');
    if (slash != std::string::npos) { sub_dir = t_match.substr(slash); t_match = t_match.substr(0, slash); }
    uint64_t dir_addr;
    if (!r.lookup(root, dir, &dir_addr)) return BMADGPU_EINVAL;
    Object dir_obj = r.object(dir_addr);
    if (!dir_obj.is_group) return BMADGPU_EINVAL;
    std::vector<std::pair<std::string, uint64_t>> ch;
    r.children(dir_obj.btree, dir_obj.heap, ch);
    std::sort(ch.begin(), ch.end());
    const size_t pt = t_match.find("%T");
    const std::string pre = t_match.substr(0, pt), post = t_match.substr(pt + 2);
    for (auto& c : ch) {
      const std::string& nm = c.first;
      if (!r.object(c.second).is_group) continue;
      if (nm.size() < pre.size() + post.size() + 1) continue;
      if (nm.compare(0, pre.size(), pre) != 0) continue;
      if (nm.compare(nm.size() - post.size(), post.size(), post) != 0) continue;
      if (!is_integer(nm.substr(pre.size(), nm.size() - pre.size() - post.size()))) continue;
      bunch_paths.push_back(dir + nm + sub_dir);
    }
  }
  if (n_bunch) *n_bunch = (int32_t)bunch_paths.size();
  if (ix_bunch < 0 || ix_bunch >= (int32_t)bunch_paths.size()) return BMADGPU_EINVAL;

  // The species group: particlesPath itself (old layout) or its first child group with numParticles.
  uint64_t bunch_addr, particles;
  if (!r.lookup(root, bunch_paths[ix_bunch], &bunch_addr)) return BMADGPU_EINVAL;
  if (!r.lookup(bunch_addr, particles_path, &particles)) return BMADGPU_EINVAL;
  uint64_t species = particles;
  Object so = r.object(particles);
  if (!so.attrs.count("numParticles")) {
    bool found = false;
    std::vector<std::pair<std::string, uint64_t>> ch;
    r.children(so.btree, so.heap, ch);
    std::sort(ch.begin(), ch.end());
    for (auto& c : ch) {
      Object g = r.object(c.second);
      if (g.is_group && g.attrs.count("numParticles")) { species = c.second; so = g; found = true; break; }
    }
    if (!found) return BMADGPU_EINVAL;
  }
  const Attr& na = so.attrs["numParticles"];
  const int64_t n = Reader::int_at(na.type, na.data);
  if (n < 0) return BMADGPU_EINVAL;
  if (!so.attrs.count("speciesType")) return BMADGPU_EINVAL;   // the reference needs the species
  if (Reader::str(so.attrs["speciesType"]) == "photon") return BMADGPU_EUNSUPPORTED;
  *n_particle = n;
  if (!b || !b->vec) return BMADGPU_OK;                        // size query
  if (b->n != n || !b->beta || !b->state) return BMADGPU_EINVAL;

  const double f_ev = kECharge / kCLight;                      // unit_eV_per_c%unitSI
  std::vector<double> v[6], off, dt(n, 0.0), t0(n, 0.0), tot_mom, p0c(n, 0.0);
  for (int i = 0; i < 6; i++) v[i].assign(n, 0.0);
  const char* ax = "xyz";
  for (int k = 0; k < 3; k++) {
    read_record(r, species, std::string("position/") + ax[k], 1.0, n, v[2 * k]);
    if (read_record(r, species, std::string("positionOffset/") + ax[k], 1.0, n, off))
      for (int64_t j = 0; j < n; j++) v[2 * k][j] += off[j];
    read_record(r, species, std::string("momentum/") + ax[k], f_ev, n, v[2 * k + 1]);
    if (read_record(r, species, std::string("momentumOffset/") + ax[k], f_ev, n, off))
      for (int64_t j = 0; j < n; j++) v[2 * k + 1][j] += off[j];
  }
  read_record(r, species, "time", 1.0, n, dt);
  read_record(r, species, "timeOffset", 1.0, n, t0);
  const bool have_tot = read_record(r, species, "totalMomentum", f_ev, n, tot_mom);
  read_record(r, species, "totalMomentumOffset", f_ev, n, p0c);
  std::vector<int64_t> state, ix_ele, loc;
  const bool have_state = read_int_record(r, species, "particleStatus", n, state);
  const bool have_ele = read_int_record(r, species, "elementIndex", n, ix_ele);
  const bool have_loc = read_int_record(r, species, "locationInElement", n, loc);

  for (int64_t j = 0; j < n; j++) {
    // p0c_initial: the file's, or the lattice's where the file has none (the reference's reading
    // with an element); p0c_final: the lattice's with an element, else p0c_initial
    // (hdf5_read_beam.f90:283-340, conserve_momentum at its default)
    const double p_init = p0c[j] != 0 ? p0c[j] : param->p0c;
    const double pc0 = at_ele ? param->p0c : p_init;
    if (pc0 == 0 || p_init == 0) return BMADGPU_EINVAL;        // reference momentum not present
    int st = have_state ? (int)state[j] : 1;
    if (st != 1 && st != 0 && software != "Bmad") st = 2;     // alive$, pre_born$ = 0 kept; others lost$ (non-Bmad files)
    double pz;
    if (!have_tot)
      pz = (std::sqrt(v[1][j] * v[1][j] + v[3][j] * v[3][j] + v[5][j] * v[5][j]) - pc0) / pc0;
    else
      pz = tot_mom[j] / p_init;
    const double pc = (1 + pz) * pc0;
    const double beta = pc / std::sqrt(pc * pc + param->mass * param->mass);   // convert_pc_to
    b->vec[0 * n + j] = v[0][j];
    b->vec[1 * n + j] = v[1][j] / pc0;
    b->vec[2 * n + j] = v[2][j];
    b->vec[3 * n + j] = v[3][j] / pc0;
    b->vec[4 * n + j] = -beta * kCLight * dt[j];
    b->vec[5 * n + j] = pz;
    b->beta[j] = beta;
    if (b->t) b->t[j] = t0[j] + dt[j];
    b->state[j] = st;
    // with an element, every particle is placed at its exit (the beginning element here)
    if (b->ix_ele) b->ix_ele[j] = have_ele && !at_ele ? (int32_t)ix_ele[j] - 1 : -1;   // Bmad's 1-based index
    if (b->location) {
      const int64_t l = have_loc && !at_ele ? loc[j] : 1;
      b->location[j] = l == -1 ? 1 : l == 0 ? 3 : 2;           // upstream_end$, inside$, downstream_end$
    }
  }
  return BMADGPU_OK;
}

// ---- writing ---------------------------------------------------------------------------------

// The file is laid out in memory and written once. Addresses are file offsets (base address 0).
class Writer {
 public:
  static constexpr int kLeafK = 4, kNodeK = 16;   // the library's defaults (symbol-table nodes of 8)

  struct Msg {
    int type;
    int flags;
    std::vector<uint8_t> body;
  };
  struct Node {                                    // a group or dataset under construction
    std::vector<Msg> msgs;
    std::vector<std::pair<std::string, int>> kids; // child name, node index
    bool group = true;
    std::vector<uint8_t> data;                     // dataset contents (contiguous)
    uint64_t oh = 0, btree = 0, heap = 0;          // addresses once placed
  };

  std::vector<Node> nodes{Node()};                 // node 0 is the root group

  int add(int parent, const std::string& name, bool group) {
    nodes.push_back(Node());
    nodes.back().group = group;
    nodes[parent].kids.push_back({name, (int)nodes.size() - 1});
    return (int)nodes.size() - 1;
  }

  static void put(std::vector<uint8_t>& v, uint64_t x, int n) {
    for (int i = 0; i < n; i++) v.push_back((uint8_t)(x >> (8 * i)));
  }
  static void pad8(std::vector<uint8_t>& v) {
    while (v.size() % 8) v.push_back(0);
  }
  static std::vector<uint8_t> type_f64() {
    std::vector<uint8_t> t = {0x11, 0x20, 0x3f, 0x00};   // float, version 1, little-endian IEEE
    put(t, 8, 4);
    put(t, 0, 2); put(t, 64, 2);                         // bit offset, precision
    t.insert(t.end(), {52, 11, 0, 52});                  // exponent location/size, mantissa location/size
    put(t, 1023, 4);                                     // exponent bias
    return t;
  }
  static std::vector<uint8_t> type_i32() {
    std::vector<uint8_t> t = {0x10, 0x08, 0x00, 0x00};   // fixed-point, version 1, signed little-endian
    put(t, 4, 4);
    put(t, 0, 2); put(t, 32, 2);
    return t;
  }
  static std::vector<uint8_t> type_str(size_t n) {
    std::vector<uint8_t> t = {0x13, 0x00, 0x00, 0x00};   // string, null-terminated ASCII
    put(t, n, 4);
    return t;
  }
  static std::vector<uint8_t> space(int64_t n) {       // version 1; n < 0: scalar
    std::vector<uint8_t> s = {1, (uint8_t)(n < 0 ? 0 : 1), (uint8_t)(n < 0 ? 0 : 1), 0};
    put(s, 0, 4);
    if (n >= 0) { put(s, n, 8); put(s, n, 8); }        // dimension and maximum dimension
    return s;
  }

  static Msg attr(const std::string& name, const std::vector<uint8_t>& type, const std::vector<uint8_t>& sp,
                  const void* data, size_t bytes) {
    Msg m{0x0C, 0, {}};
    auto& v = m.body;
    v.push_back(1); v.push_back(0);
    put(v, name.size() + 1, 2); put(v, type.size(), 2); put(v, sp.size(), 2);
    v.insert(v.end(), name.begin(), name.end()); v.push_back(0); pad8(v);
    v.insert(v.end(), type.begin(), type.end()); pad8(v);
    v.insert(v.end(), sp.begin(), sp.end()); pad8(v);
    const uint8_t* p = (const uint8_t*)data;
    v.insert(v.end(), p, p + bytes);
    pad8(v);
    return m;
  }
  void attr_str(int node, const std::string& name, const std::string& s) {
    std::vector<char> z(s.begin(), s.end());
    z.push_back(0);
    nodes[node].msgs.push_back(attr(name, type_str(z.size()), space(-1), z.data(), z.size()));
  }
  void attr_f64(int node, const std::string& name, const double* x, int64_t n) {
    nodes[node].msgs.push_back(attr(name, type_f64(), space(n), x, 8 * n));
  }
  void attr_i32(int node, const std::string& name, const int32_t* x, int64_t n) {
    nodes[node].msgs.push_back(attr(name, type_i32(), space(n), x, 4 * n));
  }

  void dataset(int node, const std::vector<uint8_t>& type, int64_t n, const void* data, size_t bytes) {
    Node& d = nodes[node];
    d.group = false;
    d.msgs.push_back({0x01, 0, space(n)});
    d.msgs.push_back({0x03, 1, type});
    d.msgs.push_back({0x05, 1, {2, 2, 2, 1, 0, 0, 0, 0}});      // fill value: late allocation, default fill
    d.data.assign((const uint8_t*)data, (const uint8_t*)data + bytes);
    d.msgs.push_back({0x08, 0, {}});                             // layout, completed when placed
  }

  std::vector<uint8_t> out;

  uint64_t alloc(size_t n) {
    const uint64_t a = out.size();
    out.resize(out.size() + (n + 7) / 8 * 8, 0);
    return a;
  }
  void poke(uint64_t at, uint64_t x, int n) {
    for (int i = 0; i < n; i++) out[at + i] = (uint8_t)(x >> (8 * i));
  }

  // Places a node and (recursively) its children; returns the object header address.
  uint64_t place(int ni) {
    Node& nd = nodes[ni];
    if (!nd.group) {
      const uint64_t da = nd.data.empty() ? kUndef : alloc(nd.data.size());
      if (!nd.data.empty()) std::memcpy(out.data() + da, nd.data.data(), nd.data.size());
      for (auto& m : nodes[ni].msgs)
        if (m.type == 0x08) {
          m.body = {3, 1};
          put(m.body, da, 8);
          put(m.body, nodes[ni].data.size(), 8);
          pad8(m.body);
        }
    } else {
      std::vector<std::pair<std::string, int>> kids = nodes[ni].kids;
      std::sort(kids.begin(), kids.end());
      std::vector<uint64_t> kid_oh(kids.size());
      for (size_t k = 0; k < kids.size(); k++) kid_oh[k] = place(kids[k].second);
      // local heap: "" at 0, then the names, each padded to 8
      std::vector<uint8_t> seg(8, 0);
      std::vector<uint64_t> name_off;
      for (auto& k : kids) {
        name_off.push_back(seg.size());
        seg.insert(seg.end(), k.first.begin(), k.first.end());
        seg.push_back(0);
        pad8(seg);
      }
      const uint64_t heap = alloc(32), seg_at = alloc(seg.size());
      std::memcpy(out.data() + heap, "HEAP", 4);
      poke(heap + 8, seg.size(), 8);
      poke(heap + 16, 1, 8);                                   // no free block (end-of-list marker)
      poke(heap + 24, seg_at, 8);
      std::memcpy(out.data() + seg_at, seg.data(), seg.size());
      // symbol-table nodes of at most 2 * kLeafK entries, one B-tree node above them
      const size_t per = 2 * kLeafK;
      const size_t n_snod = kids.empty() ? 0 : (kids.size() + per - 1) / per;
      if (n_snod > 2 * (size_t)kNodeK) throw Err{BMADGPU_EUNSUPPORTED};   // one B-tree node only
      const uint64_t tree = alloc(24 + 16 * 2 * kNodeK + 8);
      std::memcpy(out.data() + tree, "TREE", 4);
      poke(tree + 4, 0, 1); poke(tree + 5, 0, 1); poke(tree + 6, n_snod, 2);
      poke(tree + 8, kUndef, 8); poke(tree + 16, kUndef, 8);
      poke(tree + 24, 0, 8);                                   // key 0: the empty name
      for (size_t s = 0; s < n_snod; s++) {
        const uint64_t sn = alloc(8 + 40 * per);
        std::memcpy(out.data() + sn, "SNOD", 4);
        poke(sn + 4, 1, 1);
        const size_t lo = s * per, hi = std::min(kids.size(), lo + per);
        poke(sn + 6, hi - lo, 2);
        for (size_t k = lo; k < hi; k++) {
          const uint64_t e = sn + 8 + 40 * (k - lo);
          poke(e, name_off[k], 8);
          poke(e + 8, kid_oh[k], 8);
          const Node& kn = nodes[kids[k].second];
          if (kn.group) { poke(e + 16, 1, 4); poke(e + 24, kn.btree, 8); poke(e + 32, kn.heap, 8); }
        }
        poke(tree + 32 + 16 * s, sn, 8);                       // child s
        poke(tree + 40 + 16 * s, name_off[hi - 1], 8);         // key s + 1: its last name
      }
      nodes[ni].btree = tree;
      nodes[ni].heap = heap;
      Msg st{0x11, 0, {}};
      put(st.body, tree, 8);
      put(st.body, heap, 8);
      nodes[ni].msgs.push_back(st);
    }
    // version-1 object header, all messages in one block
    const Node& n2 = nodes[ni];
    size_t size = 0;
    for (auto& m : n2.msgs) size += 8 + (m.body.size() + 7) / 8 * 8;
    const uint64_t oh = alloc(16 + size);
    poke(oh, 1, 1);
    poke(oh + 2, n2.msgs.size(), 2);
    poke(oh + 4, 1, 4);
    poke(oh + 8, size, 4);
    uint64_t p = oh + 16;
    for (auto& m : n2.msgs) {
      const size_t bl = (m.body.size() + 7) / 8 * 8;
      poke(p, m.type, 2);
      poke(p + 2, bl, 2);
      poke(p + 4, m.flags, 1);
      std::memcpy(out.data() + p + 8, m.body.data(), m.body.size());
      p += 8 + bl;
    }
    nodes[ni].oh = oh;
    return oh;
  }

  std::vector<uint8_t> finish() {
    out.assign(96, 0);
    const uint64_t root_oh = place(0);
    static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    std::memcpy(out.data(), sig, 8);
    out[13] = 8; out[14] = 8;
    poke(16, kLeafK, 2); poke(18, kNodeK, 2);
    poke(24, 0, 8); poke(32, kUndef, 8); poke(40, out.size(), 8); poke(48, kUndef, 8);
    poke(56, 0, 8); poke(64, root_oh, 8); poke(72, 1, 4);
    poke(80, nodes[0].btree, 8); poke(88, nodes[0].heap, 8);
    return out;
  }
};

struct Unit {
  const char* symbol;
  double si;
  double dim[7];
};

// pmd_write_units_to_dataset: localName, unitSI, unitDimension, unitSymbol.
void units(Writer& w, int node, const char* local, const Unit& u) {
  w.attr_str(node, "localName", local);
  w.attr_f64(node, "unitSI", &u.si, 1);
  w.attr_f64(node, "unitDimension", u.dim, 7);
  w.attr_str(node, "unitSymbol", u.symbol);
}

// pmd_write_real_to_dataset_rank1: a dataset with minValue/maxValue, or a constant component.
void real_record(Writer& w, int parent, const char* name, const char* local, const Unit& u,
                 const std::vector<double>& x) {
  const int64_t n = (int64_t)x.size();
  double lo = n ? x[0] : 0, hi = lo;
  for (double v : x) { lo = std::min(lo, v); hi = std::max(hi, v); }
  if (lo == hi) {
    const int node = w.add(parent, name, true);
    const int32_t shape = (int32_t)n;
    w.attr_f64(node, "value", &hi, 1);
    w.attr_i32(node, "shape", &shape, 1);
    units(w, node, local, u);
    return;
  }
  const int node = w.add(parent, name, false);
  w.dataset(node, Writer::type_f64(), n, x.data(), 8 * x.size());
  w.attr_f64(node, "minValue", &lo, 1);
  w.attr_f64(node, "maxValue", &hi, 1);
  units(w, node, local, u);
}

void int_record(Writer& w, int parent, const char* name, const char* local, const Unit& u,
                const std::vector<int32_t>& x) {
  const int64_t n = (int64_t)x.size();
  int32_t lo = n ? x[0] : 0, hi = lo;
  for (int32_t v : x) { lo = std::min(lo, v); hi = std::max(hi, v); }
  if (lo == hi) {
    const int node = w.add(parent, name, true);
    const int32_t shape = (int32_t)n;
    w.attr_i32(node, "value", &hi, 1);
    w.attr_i32(node, "shape", &shape, 1);
    units(w, node, local, u);
    return;
  }
  const int node = w.add(parent, name, false);
  w.dataset(node, Writer::type_i32(), n, x.data(), 4 * x.size());
  w.attr_i32(node, "minValue", &lo, 1);
  w.attr_i32(node, "maxValue", &hi, 1);
  units(w, node, local, u);
}

const char* species_name(const bmadgpu_param* p) {
  const bool e = std::fabs(p->mass - 0.51099895069e6) < 1e-3 * 0.51099895069e6;
  const bool pr = std::fabs(p->mass - 0.93827208943e9) < 1e-3 * 0.93827208943e9;
  if (e) return p->charge < 0 ? "electron" : "positron";
  if (pr) return p->charge > 0 ? "proton" : "anti-proton";
  return nullptr;
}

// One bunch group "/data/<ib, i5.5>/particles/<species>/" (ib counted from 1) with its records (hdf5_write_beam.f90:95-240).
int add_bunch(Writer& w, int data, int ib, const bmadgpu_bunch* b, const bmadgpu_param* param, const char* species,
              double s_position, bool alive_only) {
  if (!b || b->n < 0 || !b->vec || !b->beta || !b->state) return BMADGPU_EINVAL;
  std::vector<int64_t> idx;
  for (int64_t j = 0; j < b->n; j++)
    if (!alive_only || b->state[j] == 1) idx.push_back(j);
  const int64_t n = (int64_t)idx.size();
  if (n == 0) return BMADGPU_EINVAL;
  auto col = [&](int i) {
    std::vector<double> c(n);
    for (int64_t k = 0; k < n; k++) c[k] = b->vec[i * b->n + idx[k]];
    return c;
  };
  const double p0c = param->p0c;   // p0c = 0 would be written as -1 by the reference
  const Unit u1{"", 1.0, {0, 0, 0, 0, 0, 0, 0}};
  const Unit um{"m", 1.0, {1, 0, 0, 0, 0, 0, 0}};
  const Unit us{"sec", 1.0, {0, 0, 1, 0, 0, 0, 0}};
  const Unit uev{"eV/c", kECharge / kCLight, {1, 1, -1, 0, 0, 0, 0}};
  const Unit uhbar{"hbar", kECharge * kHbar, {2, 1, -1, 0, 0, 0, 0}};

  char bunch_name[16];
  std::snprintf(bunch_name, sizeof bunch_name, "%05d", ib);
  const int bunch = w.add(data, bunch_name, true);
  const int parts = w.add(bunch, "particles", true);
  const int sp = w.add(parts, species, true);
  w.attr_str(sp, "speciesType", species);
  const double zero = 0, one = 1;
  w.attr_f64(sp, "totalCharge", &zero, 1);
  w.attr_f64(sp, "chargeLive", &zero, 1);
  w.attr_f64(sp, "chargeUnitSI", &one, 1);
  const int32_t np = (int32_t)n;
  w.attr_i32(sp, "numParticles", &np, 1);

  std::vector<double> x = col(0), px = col(1), y = col(2), py = col(3), z = col(4), pz = col(5);
  std::vector<double> mx(n), my(n), ms(n), mt(n), t(n), tof(n), pc(n, p0c), zeros(n, 0.0), s(n, s_position);
  for (int64_t k = 0; k < n; k++) {
    const int64_t j = idx[k];
    mx[k] = px[k] * p0c;
    my[k] = py[k] * p0c;
    ms[k] = std::sqrt((1 + pz[k]) * (1 + pz[k]) - px[k] * px[k] - py[k] * py[k]) * p0c;   // direction +1
    mt[k] = pz[k] * p0c;
    t[k] = -z[k] / (b->beta[j] * kCLight);                                             // t - t_ref
    tof[k] = (b->t ? b->t[j] : 0.0) - t[k];
  }
  const int mom = w.add(sp, "momentum", true);
  real_record(w, mom, "x", "px * p0c", uev, mx);
  real_record(w, mom, "y", "py * p0c", uev, my);
  real_record(w, mom, "z", "ps * p0c", uev, ms);
  real_record(w, sp, "totalMomentum", "pz * p0c", uev, mt);
  const int spin = w.add(sp, "spin", true);
  real_record(w, spin, "x", "Sx", uhbar, zeros);
  real_record(w, spin, "y", "Sy", uhbar, zeros);
  real_record(w, spin, "z", "Sz", uhbar, zeros);
  real_record(w, sp, "totalMomentumOffset", "p0c", uev, pc);
  real_record(w, sp, "time", "t - t_ref", us, t);
  real_record(w, sp, "timeOffset", "t_ref", us, tof);
  const int pos = w.add(sp, "position", true);
  real_record(w, pos, "x", "x", um, x);
  real_record(w, pos, "y", "y", um, y);
  real_record(w, pos, "z", "z", um, zeros);
  real_record(w, sp, "sPosition", "s", um, s);
  real_record(w, sp, "weight", "macro-charge", u1, zeros);
  std::vector<int32_t> st(n), br(n, 0), el(n), lc(n);
  for (int64_t k = 0; k < n; k++) {
    const int64_t j = idx[k];
    st[k] = b->state[j];
    el[k] = b->ix_ele && b->state[j] != 1 ? b->ix_ele[j] + 1 : 0;
    const int l = b->location ? b->location[j] : 2;
    lc[k] = l == 1 ? -1 : l == 3 ? 0 : 1;
  }
  int_record(w, sp, "particleStatus", "state", u1, st);
  int_record(w, sp, "branchIndex", "ix_branch", u1, br);
  int_record(w, sp, "elementIndex", "ix_ele", u1, el);
  int_record(w, sp, "locationInElement", "location", u1, lc);
  return BMADGPU_OK;
}

int save(const char* path, Writer& w) {
  const std::vector<uint8_t> bytes = w.finish();
  FILE* f = std::fopen(path, "wb");
  if (!f) return BMADGPU_EINVAL;
  const bool ok = std::fwrite(bytes.data(), 1, bytes.size(), f) == bytes.size();
  return std::fclose(f) == 0 && ok ? BMADGPU_OK : BMADGPU_EINVAL;
}

std::string time_stamp() {   // date_and_time_stamp's "yyyy-mm-dd hh:mm:ss"
  char stamp[32] = "";
  const std::time_t now = std::time(nullptr);
  std::tm tm_now{};
  if (localtime_r(&now, &tm_now)) std::strftime(stamp, sizeof stamp, "%Y-%m-%d %H:%M:%S", &tm_now);
  return stamp;
}

bool load_file(const char* path, std::vector<uint8_t>& bytes) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  uint8_t buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) bytes.insert(bytes.end(), buf, buf + got);
  std::fclose(f);
  return true;
}

// Copies the object at addr (a group with its subtree, or a dataset with its data) into writer
// node ni: attribute, dataspace, datatype and fill messages as they are, storage and symbol
// tables rebuilt. Objects with shared (committed) messages are not copied, nor objects reached
// twice (a second hard link, or a cycle in a damaged file).
void copy_tree(Reader& r, uint64_t addr, Writer& w, int ni, int depth, std::set<uint64_t>& seen) {
  if (depth > 32) throw Err{BMADGPU_EINVAL};
  if (!seen.insert(addr).second) throw Err{BMADGPU_EUNSUPPORTED};
  Object o = r.object(addr);
  if (o.is_group == o.is_dataset) throw Err{BMADGPU_EUNSUPPORTED};
  for (const auto& m : o.raw) {
    if (m.flags & 2) throw Err{BMADGPU_EUNSUPPORTED};                 // shared message
    if (m.type == 0x01 || m.type == 0x03 || m.type == 0x05 || m.type == 0x0C || m.type == 0x12)
      w.nodes[ni].msgs.push_back({m.type, m.flags & 1, std::vector<uint8_t>(m.body, m.body + m.size)});
  }
  if (o.is_dataset) {
    if (!o.data) throw Err{BMADGPU_EUNSUPPORTED};                     // storage never written
    w.nodes[ni].group = false;
    w.nodes[ni].data.assign(o.data, o.data + o.data_bytes);
    w.nodes[ni].msgs.push_back({0x08, 0, {}});
    return;
  }
  std::vector<std::pair<std::string, uint64_t>> ch;
  r.children(o.btree, o.heap, ch);
  for (auto& c : ch) copy_tree(r, c.second, w, w.add(ni, c.first, true), depth + 1, seen);
}

int write_hdf5(const char* path, const bmadgpu_bunch* bunches, int32_t n_bunch, const bmadgpu_param* param,
               double s_position, int32_t flags) {
  if (n_bunch < 1 || n_bunch > 2 * Writer::kLeafK * 2 * Writer::kNodeK) return BMADGPU_EINVAL;
  const char* species = species_name(param);
  if (!species) return BMADGPU_EUNSUPPORTED;
  Writer w;
  std::vector<uint8_t> old;
  if ((flags & BMADGPU_BEAM_APPEND) && load_file(path, old)) {
    // hdf5_write_beam with append: the file as it is, a lastUpdated stamp, and the new bunches under
    // the first free numbers of basePath "/data/%T/" (hdf5_write_beam.f90:43-47, 99-106)
    Reader r(std::move(old));
    const uint64_t root = r.root();
    Object ro = r.object(root);
    if (!ro.attrs.count("basePath") || Reader::str(ro.attrs["basePath"]) != "/data/%T/") return BMADGPU_EUNSUPPORTED;
    std::set<uint64_t> seen;
    copy_tree(r, root, w, 0, 0, seen);
    auto& rm = w.nodes[0].msgs;
    const std::string stamp = time_stamp();
    rm.erase(std::remove_if(rm.begin(), rm.end(), [](const Writer::Msg& m) {
               return m.type == 0x0C && m.body.size() > 8 + 11 && std::memcmp(m.body.data() + 8, "lastUpdated", 12) == 0;
             }), rm.end());
    w.attr_str(0, "lastUpdated", stamp);
    int data = -1;
    for (auto& k : w.nodes[0].kids)
      if (k.first == "data") data = k.second;
    if (data < 0 || !w.nodes[data].group) return BMADGPU_EINVAL;
    int number = 0;
    for (int32_t ib = 0; ib < n_bunch; ib++) {
      bool taken = true;
      while (taken) {
        char nm[16];
        std::snprintf(nm, sizeof nm, "%05d", ++number);
        taken = false;
        for (auto& k : w.nodes[data].kids) taken = taken || k.first == nm;
      }
      if (w.nodes[data].kids.size() >= (size_t)(2 * Writer::kLeafK * 2 * Writer::kNodeK)) return BMADGPU_EINVAL;
      const int rr = add_bunch(w, data, number, &bunches[ib], param, species, s_position,
                               (flags & BMADGPU_BEAM_ALIVE_ONLY) != 0);
      if (rr) return rr;
    }
    return save(path, w);
  }
  w.attr_str(0, "dataType", "openPMD");
  w.attr_str(0, "openPMD", "2.0.0");
  w.attr_str(0, "openPMDextension", "BeamPhysics;SpeciesType");
  w.attr_str(0, "basePath", "/data/%T/");
  w.attr_str(0, "particlesPath", "particles/");
  w.attr_str(0, "software", "Bmad");
  w.attr_str(0, "softwareVersion", "1.0");
  w.attr_str(0, "date", time_stamp());
  const int data = w.add(0, "data", true);
  for (int32_t ib = 0; ib < n_bunch; ib++) {
    const int r = add_bunch(w, data, ib + 1, &bunches[ib], param, species, s_position,
                            (flags & BMADGPU_BEAM_ALIVE_ONLY) != 0);
    if (r) return r;
  }

  return save(path, w);
}

}  // namespace

extern "C" int bmadgpu_beam_write_hdf5(const char* path, const bmadgpu_bunch* host_bunch, const bmadgpu_param* param,
                                       double s_position, int32_t flags) {
  if (!path || !host_bunch || !param) return BMADGPU_EINVAL;
  try {
    return write_hdf5(path, host_bunch, 1, param, s_position, flags);
  } catch (const Err& e) {
    return e.code;
  }
}

extern "C" int bmadgpu_beam_write_hdf5_bunches(const char* path, const bmadgpu_bunch* host_bunches, int32_t n_bunch,
                                               const bmadgpu_param* param, double s_position, int32_t flags) {
  if (!path || !host_bunches || !param) return BMADGPU_EINVAL;
  try {
    return write_hdf5(path, host_bunches, n_bunch, param, s_position, flags);
  } catch (const Err& e) {
    return e.code;
  }
}

extern "C" int bmadgpu_beam_read_hdf5(const char* path, const bmadgpu_param* param, int32_t ix_bunch, int32_t flags,
                                      bmadgpu_bunch* host_bunch, int64_t* n_particle, int32_t* n_bunch) {
  if (!path || !param || !n_particle) return BMADGPU_EINVAL;
  try {
    return read_hdf5(path, param, ix_bunch, flags, host_bunch, n_particle, n_bunch);
  } catch (const Err& e) {
    return e.code;
  }
}

// write_beam_file / read_beam_file (bmad/multiparticle/beam_file_io.f90:29-106, 380-420): the file
// name picks the format, HDF5 for names ending in ".h5" or ".hdf5", else Bmad's ASCII layout.
static bool is_hdf5_name(const char* path) {
  const size_t n = std::strlen(path);
  return (n > 3 && std::strcmp(path + n - 3, ".h5") == 0) || (n > 5 && std::strcmp(path + n - 5, ".hdf5") == 0);
}

extern "C" int bmadgpu_beam_write_file(const char* path, const bmadgpu_bunch* host_bunch, const bmadgpu_param* param,
                                       double s_position, int32_t flags) {
  if (!path) return BMADGPU_EINVAL;
  if (is_hdf5_name(path))   // doubles are stored as they are: BMADGPU_BEAM_EXACT has nothing to add
    return bmadgpu_beam_write_hdf5(path, host_bunch, param, s_position, flags & ~BMADGPU_BEAM_EXACT);
  return bmadgpu_beam_write_ascii(path, host_bunch, param, s_position, flags);
}

extern "C" int bmadgpu_beam_read_file(const char* path, const bmadgpu_param* param, bmadgpu_bunch* host_bunch,
                                      int64_t* n_particle) {
  if (!path) return BMADGPU_EINVAL;
  if (is_hdf5_name(path)) return bmadgpu_beam_read_hdf5(path, param, 0, 0, host_bunch, n_particle, nullptr);
  return bmadgpu_beam_read_ascii(path, param, host_bunch, n_particle);
}
