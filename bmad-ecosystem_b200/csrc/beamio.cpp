// beamio.cpp -- Bmad's ASCII beam file (version 4) for checkpoint and resume.
//
// Writer: write_ascii_beam_file (bmad/multiparticle/beam_file_io.f90:112-300): per bunch a
// header of "# key = value" lines (counts, then the per-particle fields that are the same for
// every particle), a "#!" line naming the columns, and one line per particle. The columns written
// are those of the reference for a tracked bunch without fields, phase or per-particle charge:
// index, x px y py z pz, p0c, s_position, time, spin_x spin_y spin_z, state, ix_ele, location;
// numbers in es23.15, the same formats as the reference (i8, a14, a16). With BMADGPU_BEAM_EXACT
// the numbers carry 17 significant digits (es24.16) and a beta column (a column the reference's
// reader accepts) is added, so that a run resumed from the file continues bit for bit.
// Reader: read_beam_ascii (beam_file_io.f90:834-1282) for such files: header values, the column
// list, then the rows; columns it does not need are skipped by name. Files of the older
// "!ASCII::3" layout (read_beam_file, beam_file_io.f90:500-620: a BEGIN_BUNCH block with species,
// charge, z and t centres, then rows of vec(6), charge, state, spin(3), ix_ele, location) are read
// too; only their first bunch is used.

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include <strings.h>

#include "../../include/bmadgpu.h"

namespace {

std::string es(int w, int d, double x) {  // Fortran ESw.d
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.*E", d, x);
  std::string s(buf);
  size_t e = s.find('E');
  int ev = std::atoi(s.c_str() + e + 1);
  char eb[16];
  if (std::abs(ev) < 100) std::snprintf(eb, sizeof eb, "E%c%02d", ev < 0 ? '-' : '+', std::abs(ev));
  else std::snprintf(eb, sizeof eb, "%c%03d", ev < 0 ? '-' : '+', std::abs(ev));
  s = s.substr(0, e) + eb;
  if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
  return s;
}

std::string rpad(int w, const std::string& s) {  // Fortran a<w>: right-justified
  return (int)s.size() >= w ? s : std::string(w - s.size(), ' ') + s;
}

const char* state_name(int st) {  // coord_state_name, bmad/modules/bmad_struct.f90:2635-2659
  switch (st) {
    case 1: return "Alive";
    case 2: return "Lost";
    case 3: return "Lost_Neg_X";
    case 4: return "Lost_Pos_X";
    case 5: return "Lost_Neg_Y";
    case 6: return "Lost_Pos_Y";
    case 7: return "Lost_Z";
    case 8: return "Lost_Pz";
    case 0: return "Pre_Born";
    default: return "Not_Set";
  }
}

int state_id(const std::string& s) {
  static const char* names[] = {"Pre_Born", "Alive", "Lost", "Lost_Neg_X", "Lost_Pos_X",
                                "Lost_Neg_Y", "Lost_Pos_Y", "Lost_Z", "Lost_Pz"};
  for (int i = 0; i < 9; i++)
    if (strcasecmp(s.c_str(), names[i]) == 0) return i;
  return -999;
}

const char* location_name(int loc) {  // bmad_struct.f90:403-404
  switch (loc) {
    case 1: return "Upstream_End";
    case 2: return "Downstream_End";
    case 3: return "Inside";
    default: return "GARBAGE!";
  }
}

int location_id(const std::string& s) {
  if (strcasecmp(s.c_str(), "Upstream_End") == 0) return 1;
  if (strcasecmp(s.c_str(), "Downstream_End") == 0) return 2;
  if (strcasecmp(s.c_str(), "Inside") == 0) return 3;
  return 0;
}

const char* species_name(const bmadgpu_param& p) {
  // the species of the configurations this path serves (electrons and positrons)
  return p.charge < 0 ? "Electron" : "Positron";
}

// A real as Fortran writes it: also "1.234567-100" (three-digit exponent without the E).
double parse_real(const std::string& tok) {
  std::string t = tok;
  for (size_t i = 1; i < t.size(); i++)
    if ((t[i] == '-' || t[i] == '+') && std::isdigit((unsigned char)t[i - 1])) {
      t.insert(i, "E");
      break;
    }
  return std::strtod(t.c_str(), nullptr);
}

}  // namespace

extern "C" int bmadgpu_beam_write_ascii(const char* path, const bmadgpu_bunch* b, const bmadgpu_param* param,
                                        double s_position, int32_t flags) {
  if (!path || !b || !param || b->n < 0 || (b->n > 0 && (!b->vec || !b->state))) return BMADGPU_EINVAL;
  const bool alive_only = flags & BMADGPU_BEAM_ALIVE_ONLY, exact = flags & BMADGPU_BEAM_EXACT;
  const int W = exact ? 24 : 23, D = exact ? 16 : 15;
  FILE* f = std::fopen(path, (flags & BMADGPU_BEAM_APPEND) ? "a" : "w");
  if (!f) return BMADGPU_EINVAL;
  const int64_t n = b->n;
  int64_t n_alive = 0;
  for (int64_t j = 0; j < n; j++) n_alive += (b->state[j] == 1 || b->state[j] == 0);
  bool loc0 = true;
  for (int64_t j = 1; j < n; j++)
    if (b->location && b->location[j] != b->location[0]) loc0 = false;
  const int loc_first = (n > 0 && b->location) ? b->location[0] : 2;
  std::fprintf(f, "# ix_bunch       =%6d\n", 1);
  std::fprintf(f, "# n_particle     =%6lld\n", (long long)n);
  std::fprintf(f, "# n_alive        =%6lld\n", (long long)n_alive);
  std::fprintf(f, "# n_dead         =%6lld\n", (long long)(n - n_alive));
  // headwrite_re / _int / _str: '# ', name, tab to column 18, '=' then the value
  std::fprintf(f, "# %-15s=%s\n", "charge", es(24, 16, 0.0).c_str());
  std::fprintf(f, "# %-15s= %d\n", "ix_branch", 0);
  std::fprintf(f, "# %-15s= %d\n", "direction", 1);
  std::fprintf(f, "# %-15s= %d\n", "time_dir", 1);
  std::fprintf(f, "# %-15s= %s\n", "species", species_name(*param));
  if (loc0) std::fprintf(f, "# %-15s= %s\n", "location", location_name(loc_first));
  std::string line = rpad(8, "index");
  const char* vn[] = {"x", "px", "y", "py", "z", "pz"};
  for (int i = 0; i < 6; i++) line += rpad(W, vn[i]);
  line += rpad(W, "p0c") + rpad(W, "s_position") + rpad(W, "time");
  line += rpad(W, "spin_x") + rpad(W, "spin_y") + rpad(W, "spin_z");
  line += rpad(14, "state") + rpad(8, "ix_ele") + rpad(16, "location");
  if (exact) line += rpad(W, "beta");
  line[0] = '#';
  line[1] = '!';
  std::fprintf(f, "%s\n", line.c_str());
  for (int64_t j = 0; j < n; j++) {
    const int st = b->state[j];
    if (alive_only && st != 1 && st != 0) continue;
    char ib[32];
    std::snprintf(ib, sizeof ib, "%8lld", (long long)(j + 1));
    std::string l = ib;
    for (int i = 0; i < 6; i++) l += es(W, D, b->vec[i * n + j]);
    l += es(W, D, param->p0c) + es(W, D, s_position) + es(W, D, b->t ? b->t[j] : 0.0);
    l += es(W, D, 0.0) + es(W, D, 0.0) + es(W, D, 0.0);
    l += rpad(14, state_name(st));
    // ix_ele: the element of the loss for lost particles (1-based, as Bmad's element indices are
    // counted from the beginning element 0), else the end of the lattice
    std::snprintf(ib, sizeof ib, "%8d", b->ix_ele ? b->ix_ele[j] + 1 : 0);
    l += ib;
    l += rpad(16, location_name(b->location ? b->location[j] : 2));
    if (exact) l += es(W, D, b->beta ? b->beta[j] : 0.0);
    std::fprintf(f, "%s\n", l.c_str());
  }
  std::fclose(f);
  return BMADGPU_OK;
}

extern "C" int bmadgpu_beam_read_ascii(const char* path, const bmadgpu_param* param, bmadgpu_bunch* b,
                                       int64_t* n_particle) {
  if (!path || !n_particle || !param) return BMADGPU_EINVAL;
  std::ifstream in(path);
  if (!in) return BMADGPU_EINVAL;
  std::vector<std::string> cols;
  std::string line;
  int default_loc = 2;
  std::vector<std::vector<std::string>> rows;
  std::string first;
  std::getline(in, first);
  const bool old_layout = first.compare(0, 9, "!ASCII::3") == 0;
  if (old_layout) {
    // old layout: three header numbers, then BEGIN_BUNCH, species, three numbers, rows, END_BUNCH
    int stage = 0;
    while (std::getline(in, line)) {
      std::istringstream ss(line);
      std::string w;
      ss >> w;
      if (w.empty()) continue;
      if (stage == 0) {
        if (strcasecmp(w.c_str(), "BEGIN_BUNCH") == 0) stage = 1;
        continue;
      }
      if (stage >= 1 && stage <= 4) {  // species, charge_tot, z_center, t_center
        stage++;
        continue;
      }
      if (strcasecmp(w.c_str(), "END_BUNCH") == 0) break;
      std::vector<std::string> r{w};
      while (ss >> w) r.push_back(w);
      rows.push_back(r);
    }
    cols = {"x", "px", "y", "py", "z", "pz", "charge", "state_id", "spin_x", "spin_y", "spin_z", "ix_ele", "location_id"};
  } else {
    in.clear();
    in.seekg(0);
  }
  while (!old_layout && std::getline(in, line)) {
    if (line.empty()) continue;
    if (line.compare(0, 2, "#!") == 0) {
      std::istringstream ss(line.substr(2));
      std::string c;
      while (ss >> c) cols.push_back(c);
      continue;
    }
    if (line[0] == '#') {
      size_t eq = line.find('=');
      if (eq != std::string::npos) {
        std::istringstream kk(line.substr(1, eq - 1)), vv(line.substr(eq + 1));
        std::string key, val;
        kk >> key;
        vv >> val;
        if (strcasecmp(key.c_str(), "location") == 0) default_loc = location_id(val);
      }
      continue;
    }
    std::istringstream ss(line);
    std::vector<std::string> r;
    std::string w;
    while (ss >> w) r.push_back(w);
    if (!r.empty()) rows.push_back(r);
  }
  if (cols.empty()) return BMADGPU_EINVAL;
  // column index of each field (the vec names x..pz each take one column)
  auto find = [&](const char* name) -> int {
    for (size_t i = 0; i < cols.size(); i++)
      if (strcasecmp(cols[i].c_str(), name) == 0) return (int)i;
    return -1;
  };
  const int ix_vec[6] = {find("x"), find("px"), find("y"), find("py"), find("z"), find("pz")};
  for (int i = 0; i < 6; i++)
    if (ix_vec[i] < 0) return BMADGPU_EINVAL;
  const int ix_p0c = find("p0c"), ix_t = find("time"), ix_state = find("state"), ix_ele = find("ix_ele"),
            ix_loc = find("location"), ix_beta = find("beta"), ix_state_num = find("state_id"),
            ix_loc_num = find("location_id");
  const int64_t n = (int64_t)rows.size();
  *n_particle = n;
  if (!b || !b->vec) return BMADGPU_OK;   // size query
  if (b->n != n || !b->beta || !b->state) return BMADGPU_EINVAL;
  for (int64_t j = 0; j < n; j++) {
    const std::vector<std::string>& r = rows[j];
    if ((int)r.size() < (int)cols.size()) return BMADGPU_EINVAL;
    for (int i = 0; i < 6; i++) b->vec[i * n + j] = parse_real(r[ix_vec[i]]);
    const double p0c = ix_p0c >= 0 ? parse_real(r[ix_p0c]) : param->p0c;
    if (b->t) b->t[j] = ix_t >= 0 ? parse_real(r[ix_t]) : 0.0;
    b->state[j] = ix_state >= 0 ? state_id(r[ix_state]) : ix_state_num >= 0 ? std::atoi(r[ix_state_num].c_str()) : 1;
    if (b->ix_ele) b->ix_ele[j] = ix_ele >= 0 ? std::atoi(r[ix_ele].c_str()) - 1 : -1;
    if (b->location)
      b->location[j] = ix_loc >= 0 ? location_id(r[ix_loc])
                                   : ix_loc_num >= 0 ? std::atoi(r[ix_loc_num].c_str()) : default_loc;
    if (ix_beta >= 0) {
      b->beta[j] = parse_real(r[ix_beta]);
    } else {  // as init_coord sets it from the momentum
      const double pc = p0c * (1 + b->vec[5 * n + j]);
      b->beta[j] = pc / std::sqrt(pc * pc + param->mass * param->mass);
    }
  }
  return BMADGPU_OK;
}
