// data_file.cpp -- LAMMPS data reader with RBMD's conventions (see data_file.hpp).
#include "data_file.hpp"

#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>

namespace rbmd_host {

namespace {

bool blank(const std::string& s) {
  for (char c : s)
    if (c != ' ' && c != '\t' && c != '\r') return false;
  return true;
}

// Reads `count` non-blank lines after a section title (the reference skips blank lines the same
// way, e.g. Masses(), :280-299) and hands each to `fn`.
template <class F>
void section(std::ifstream& f, int count, const std::string& path, const std::string& name, F&& fn) {
  std::string line;
  int got = 0;
  while (got < count && std::getline(f, line)) {
    if (blank(line)) continue;
    std::istringstream iss(line);
    if (!fn(iss)) throw std::runtime_error(path + ": malformed line in " + name + ": " + line);
    ++got;
  }
  if (got < count) throw std::runtime_error(path + ": " + name + " ends after " + std::to_string(got) + " of " +
                                            std::to_string(count) + " lines");
}

int checked_id(long v, int n, const std::string& path, const std::string& what) {
  if (v < 1 || v > n) throw std::runtime_error(path + ": " + what + " id " + std::to_string(v) + " out of range");
  return (int)(v - 1);
}

}  // namespace

DataFile read_data_file(const std::string& path, const std::string& atom_style, const std::string& unit) {
  if (atom_style != "atomic" && atom_style != "charge" && atom_style != "full")
    throw std::runtime_error("atom_style must be atomic, charge or full, not \"" + atom_style + "\"");
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open data file " + path);
  DataFile d;
  std::string line;
  // header (Header(), :120-222): counts and box until the first section title
  std::getline(f, line);  // title line
  std::streampos body = f.tellg();
  while (std::getline(f, line)) {
    std::istringstream iss(line);
    if (line.find("xlo xhi") != std::string::npos) {
      iss >> d.lo[0] >> d.hi[0];
    } else if (line.find("ylo yhi") != std::string::npos) {
      iss >> d.lo[1] >> d.hi[1];
    } else if (line.find("zlo zhi") != std::string::npos) {
      iss >> d.lo[2] >> d.hi[2];
    } else if (line.find("atom types") != std::string::npos) {
      iss >> d.n_types;
    } else if (line.find("bond types") != std::string::npos) {
      iss >> d.n_bond_types;
    } else if (line.find("angle types") != std::string::npos) {
      iss >> d.n_angle_types;
    } else if (line.find("dihedral types") != std::string::npos) {
      iss >> d.n_dihedral_types;
    } else if (line.find("dihedrals") != std::string::npos) {
      iss >> d.n_dihedrals;
    } else if (line.find("atoms") != std::string::npos) {
      iss >> d.n_atoms;
    } else if (line.find("bonds") != std::string::npos) {
      iss >> d.n_bonds;
    } else if (line.find("angles") != std::string::npos) {
      iss >> d.n_angles;
    } else if (line.find("Masses") != std::string::npos || line.find("Atoms") != std::string::npos ||
               line.find("Coeffs") != std::string::npos) {
      break;
    }
    body = f.tellg();
  }
  if (d.n_atoms <= 0 || d.n_types <= 0) throw std::runtime_error(path + ": header gives no atoms or atom types");
  const int n = d.n_atoms;
  d.type_mass.assign(d.n_types, 1.0);
  d.type_eps.assign(d.n_types, 1.0);
  d.type_sigma.assign(d.n_types, 1.0);
  d.position.assign(3 * (size_t)n, 0.0);
  d.charge.assign(n, 0.0);
  d.type.assign(n, 0);
  d.molecule.resize(n);
  for (int i = 0; i < n; ++i) d.molecule[i] = i;
  std::vector<char> seen(n, 0);

  f.clear();
  f.seekg(body);
  bool have_atoms = false;
  while (std::getline(f, line)) {
    if (line.find("Masses") != std::string::npos) {
      section(f, d.n_types, path, "Masses", [&](std::istringstream& s) {
        long t;
        double m;
        if (!(s >> t >> m)) return false;
        d.type_mass[checked_id(t, d.n_types, path, "type")] = m;
        return true;
      });
      if (unit == "LJ") d.type_mass.assign(d.n_types, 1.0);
    } else if (line.find("Pair Coeffs") != std::string::npos) {
      section(f, d.n_types, path, "Pair Coeffs", [&](std::istringstream& s) {
        long t;
        double e, sg;
        if (!(s >> t >> e >> sg)) return false;
        const int k = checked_id(t, d.n_types, path, "type");
        d.type_eps[k] = e;
        d.type_sigma[k] = sg;
        return true;
      });
    } else if (line.find("Bond Coeffs") != std::string::npos) {
      d.bond_k.assign(d.n_bond_types, 0.0);
      d.bond_r0.assign(d.n_bond_types, 0.0);
      section(f, d.n_bond_types, path, "Bond Coeffs", [&](std::istringstream& s) {
        long t;
        double k, r0;
        if (!(s >> t >> k >> r0)) return false;
        const int b = checked_id(t, d.n_bond_types, path, "bond type");
        d.bond_k[b] = k;
        d.bond_r0[b] = r0;
        return true;
      });
    } else if (line.find("Angle Coeffs") != std::string::npos) {
      d.angle_k.assign(d.n_angle_types, 0.0);
      d.angle_theta0.assign(d.n_angle_types, 0.0);
      section(f, d.n_angle_types, path, "Angle Coeffs", [&](std::istringstream& s) {
        long t;
        double k, t0;
        if (!(s >> t >> k >> t0)) return false;
        const int a = checked_id(t, d.n_angle_types, path, "angle type");
        d.angle_k[a] = k;
        d.angle_theta0[a] = t0;
        return true;
      });
    } else if (line.find("Dihedral Coeffs") != std::string::npos) {
      d.dihedral_k.assign(d.n_dihedral_types, 0.0);
      d.dihedral_sign.assign(d.n_dihedral_types, 1);
      d.dihedral_multiplicity.assign(d.n_dihedral_types, 0);
      section(f, d.n_dihedral_types, path, "Dihedral Coeffs", [&](std::istringstream& s) {
        long t;
        double k;
        int sign, mult;
        if (!(s >> t >> k >> sign >> mult)) return false;
        const int a = checked_id(t, d.n_dihedral_types, path, "dihedral type");
        d.dihedral_k[a] = k;
        d.dihedral_sign[a] = sign;
        d.dihedral_multiplicity[a] = mult;
        return true;
      });
    } else if (line.find("Atoms") != std::string::npos) {
      section(f, n, path, "Atoms", [&](std::istringstream& s) {
        long id, mol = 0, t;
        double q = 0.0, x, y, z;
        if (atom_style == "atomic") {
          if (!(s >> id >> t >> x >> y >> z)) return false;
        } else if (atom_style == "charge") {
          if (!(s >> id >> t >> q >> x >> y >> z)) return false;
        } else {
          if (!(s >> id >> mol >> t >> q >> x >> y >> z)) return false;
        }
        const int i = checked_id(id, n, path, "atom");
        seen[i] = 1;
        d.type[i] = checked_id(t, d.n_types, path, "type");
        d.charge[i] = q;
        d.position[3 * (size_t)i] = x;
        d.position[3 * (size_t)i + 1] = y;
        d.position[3 * (size_t)i + 2] = z;
        if (atom_style == "full") {
          if (mol < 1) throw std::runtime_error(path + ": molecule id " + std::to_string(mol) + " out of range");
          d.molecule[i] = (int)(mol - 1);
        }
        return true;
      });
      have_atoms = true;
    } else if (line.find("Velocities") != std::string::npos) {
      d.velocity.assign(3 * (size_t)n, 0.0);
      section(f, n, path, "Velocities", [&](std::istringstream& s) {
        long id;
        double vx, vy, vz;
        if (!(s >> id >> vx >> vy >> vz)) return false;
        const int i = checked_id(id, n, path, "atom");
        d.velocity[3 * (size_t)i] = vx;
        d.velocity[3 * (size_t)i + 1] = vy;
        d.velocity[3 * (size_t)i + 2] = vz;
        return true;
      });
    } else if (line.find("Bonds") != std::string::npos) {
      d.bond_atoms.clear();
      d.bond_type.clear();
      section(f, d.n_bonds, path, "Bonds", [&](std::istringstream& s) {
        long id, t, a, b;
        if (!(s >> id >> t >> a >> b)) return false;
        d.bond_type.push_back(checked_id(t, d.n_bond_types, path, "bond type"));
        d.bond_atoms.push_back(checked_id(a, n, path, "atom"));
        d.bond_atoms.push_back(checked_id(b, n, path, "atom"));
        return true;
      });
    } else if (line.find("Dihedrals") != std::string::npos) {
      d.dihedral_atoms.clear();
      d.dihedral_type.clear();
      d.has_dihedrals = true;
      section(f, d.n_dihedrals, path, "Dihedrals", [&](std::istringstream& s) {
        long id, t, a, b, c, e;
        if (!(s >> id >> t >> a >> b >> c >> e)) return false;
        d.dihedral_type.push_back(checked_id(t, d.n_dihedral_types, path, "dihedral type"));
        for (long x : {a, b, c, e}) d.dihedral_atoms.push_back(checked_id(x, n, path, "atom"));
        return true;
      });
    } else if (line.find("Angles") != std::string::npos) {
      d.angle_atoms.clear();
      d.angle_type.clear();
      section(f, d.n_angles, path, "Angles", [&](std::istringstream& s) {
        long id, t, a, b, c;
        if (!(s >> id >> t >> a >> b >> c)) return false;
        d.angle_type.push_back(checked_id(t, d.n_angle_types, path, "angle type"));
        d.angle_atoms.push_back(checked_id(a, n, path, "atom"));
        d.angle_atoms.push_back(checked_id(b, n, path, "atom"));
        d.angle_atoms.push_back(checked_id(c, n, path, "atom"));
        return true;
      });
    }
  }
  if (!have_atoms) throw std::runtime_error(path + ": no Atoms section");
  for (int i = 0; i < n; ++i)
    if (!seen[i]) throw std::runtime_error(path + ": atom id " + std::to_string(i + 1) + " missing from Atoms");
  return d;
}

void special_lists(int n_atoms, const std::vector<int>& bond_atoms, const double weights[3], std::vector<int>& offsets,
                   std::vector<int>& ids, std::vector<double>& w) {
  std::multimap<int, int> link;  // equal keys keep insertion order
  for (size_t b = 0; b + 1 < bond_atoms.size(); b += 2) {
    link.insert({bond_atoms[b], bond_atoms[b + 1]});
    link.insert({bond_atoms[b + 1], bond_atoms[b]});
  }
  offsets.assign(1, 0);
  ids.clear();
  w.clear();
  for (int i = 0; i < n_atoms; ++i) {
    if (link.find(i) == link.end()) {
      ids.push_back(i);
      w.push_back(1.0);
      offsets.push_back((int)ids.size());
      continue;
    }
    auto r1 = link.equal_range(i);
    for (auto a = r1.first; a != r1.second; ++a) {
      const int k1 = a->second;
      ids.push_back(k1);
      w.push_back(weights[0]);
      auto r2 = link.equal_range(k1);
      for (auto b = r2.first; b != r2.second; ++b) {
        const int k2 = b->second;
        if (k2 == i) continue;
        ids.push_back(k2);
        w.push_back(weights[1]);
        auto r3 = link.equal_range(k2);
        for (auto c = r3.first; c != r3.second; ++c) {
          const int k3 = c->second;
          if (k3 == k1) continue;
          ids.push_back(k3);
          w.push_back(weights[2]);
        }
      }
    }
    offsets.push_back((int)ids.size());
  }
}

}  // namespace rbmd_host
