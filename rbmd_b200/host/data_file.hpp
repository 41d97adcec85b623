// data_file.hpp -- LAMMPS data files as RBMD reads them (read_data init configuration).
#pragma once

#include <string>
#include <vector>

namespace rbmd_host {

// The fields ModelFileInitCondition fills (framework/InitCondition/ModelFileInitCondition.cpp),
// indexed by atom id - 1 and type id - 1.
struct DataFile {
  int n_atoms = 0, n_types = 0;
  int n_bonds = 0, n_bond_types = 0, n_angles = 0, n_angle_types = 0, n_dihedrals = 0, n_dihedral_types = 0;
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  std::vector<double> type_mass;             // Masses (LJ units: all 1, Masses():296-299)
  std::vector<double> type_eps, type_sigma;  // Pair Coeffs: id eps sigma
  std::vector<double> bond_k, bond_r0;       // Bond Coeffs: id k r0
  std::vector<double> angle_k, angle_theta0; // Angle Coeffs: id k theta0 (degrees)
  std::vector<double> position;              // [3n]
  std::vector<double> velocity;              // [3n]; empty when the file has no Velocities
  std::vector<double> charge;                // [n] (0 for atom_style atomic)
  std::vector<int> type;                     // [n] 0-based
  std::vector<int> molecule;                 // [n] 0-based (full); atom i is molecule i otherwise
  std::vector<int> bond_atoms, bond_type;    // [2 nb], [nb] 0-based
  std::vector<int> angle_atoms, angle_type;  // [3 na], [na] 0-based
  // Dihedral Coeffs: id K d n (DihedralsCoeffs(), :359-376); Dihedrals: id type i j k l (:551-585)
  std::vector<double> dihedral_k;
  std::vector<int> dihedral_sign, dihedral_multiplicity;
  std::vector<int> dihedral_atoms, dihedral_type;  // [4 nd], [nd] 0-based
  bool has_dihedrals = false;                      // a Dihedrals section was read (PARA_FILE_DIHEDRALS)
};

// Reads `path` with atom_style "atomic", "charge" or "full" (Atoms(), :406-479); the unit decides
// the masses ("LJ": all 1).  Image flags at the ends of Atoms lines are ignored, as the reference
// ignores them.  Throws std::runtime_error with the file name and the offending section.
DataFile read_data_file(const std::string& path, const std::string& atom_style, const std::string& unit);

// special_ids/weights/offsets as SetSpecialBonds builds them (:848-923): per atom its 1-2, 1-3 and
// 1-4 partners through the symmetric multimap of the bond list in insertion order, weighted
// special_bonds[0..2]; an atom without bonds lists itself with weight 1.  offsets has n + 1 entries.
void special_lists(int n_atoms, const std::vector<int>& bond_atoms, const double weights[3], std::vector<int>& offsets,
                   std::vector<int>& ids, std::vector<double>& w);

}  // namespace rbmd_host
