// dynLattice input surface: .pro property files and the meshes they name.
//
// A .pro file is a JEM property file: `key.path = value;`, `key += value;`,
// `include "file";`, values are numbers, "strings", true/false, [arrays],
// references to other keys (copied, whole subtrees included) and { blocks }.
// Strings may hold $(key) substitutions and numeric expressions.  From the
// properties this module builds the engine's model description: the rod
// mesh (GMSHInput: a .geo subset meshed here, or a .msh file), node groups
// (GroupInput), the specialCosseratRod material of the Lattice model, rod
// and joint contact, the boundary-condition models (Dirichlet, Neumann,
// LoadScale, InitLoad) and added point masses (Mass), the explicit module
// (LeapFrog or MilneDevice), the run length (control.runWhile) and the output
// modules.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/dynlattice.h"

namespace dl {

// One output module of the .pro file (Output.<name>)
struct ProOutput {
  std::string name, type;                 // GroupOutput, Sample, CSVOutput, ParaView
  std::string file;                       // Sample / CSVOutput
  std::string separator = " ";            // Sample
  std::string when;                       // sampleWhen / saveWhen ("" = every step)
  std::vector<std::string> data_sets;     // Sample
  std::vector<std::string> node_groups;   // GroupOutput
  std::vector<std::string> dofs;          // GroupOutput
  std::vector<std::string> vectors;       // CSVOutput: "<vector> = <label>"
  std::string format;                     // ParaView output_format
  std::vector<std::string> node_data;     // ParaView: fint, fext, fres
  std::vector<std::string> el_data;       // ParaView: element tables (strain, stress, ...)
};

struct ProModel {
  // storage of everything `desc` points to
  std::vector<double> coords;
  std::vector<int32_t> conn, elem_rod;
  std::vector<dl_material_desc> mats;
  std::vector<std::string> strings;            // yield expressions, scale functions
  std::vector<std::vector<const char *>> derivs;
  std::vector<std::vector<double>> kin;        // kinematic tensors
  std::vector<std::vector<int32_t>> bc_nodes;
  std::vector<dl_bc_desc> bcs;
  std::vector<int32_t> given_nodes;
  std::vector<int32_t> joints;                 // joint contact: nodes of the "points" group
  std::vector<int32_t> ties;                   // rigid hinges: (original, copy) node pairs
  std::vector<double> given_dirs;
  std::vector<std::string> dof_names;
  std::vector<const char *> dof_ptrs;
  dl_model_desc desc{};
  // node groups (GroupInput and "all"), node indices
  std::map<std::string, std::vector<int32_t>> groups;
  int64_t steps = -1;    // from control.runWhile ("t <= T" or "i <= N"), -1 if not given
  double t_end = -1.0;   // end time of a time-based control.runWhile, -1 if not given
  dl_integrator_desc integ{};  // the explicit module (LeapFrog or MilneDevice)
  std::string case_name;
  std::vector<std::string> notes;  // properties read but not used by the engine
  std::vector<ProOutput> outputs;  // Output.modules, in order
};

// MilneDevice tolerance when the .pro file gives none: the reference takes
// jive::solver::Solver::PRECISION, a JIVE constant not visible here.
constexpr double kDefaultMilnePrecision = 1e-6;

// Parse `path` and everything it includes and names; throws std::runtime_error
// (message with file and line) on malformed input or unsupported features.
std::unique_ptr<ProModel> load_pro(const std::string &path);

// A .geo subset (Point, Line, DefineConstant, variables; onelab overrides)
// meshed like gmsh meshes 1D curves: `order` 1 or 2.  Outputs node
// coordinates, per line entity in tag order its elements, and the node of
// each point entity in tag order (gmsh's point elements: one per Point).
void mesh_geo(const std::string &path, int order, const std::map<std::string, double> &onelab,
              std::vector<double> &coords, std::vector<std::vector<int32_t>> &line_elems, int &nen,
              std::vector<int32_t> &point_nodes);

// gmsh .msh reader (formats 2.2 and 4.1, ASCII): 2-node and 3-node lines,
// grouped by their curve entity, and the nodes of the point elements (type
// 15) in file order.
void read_msh(const std::string &path, std::vector<double> &coords, std::vector<std::vector<int32_t>> &line_elems,
              int &nen, std::vector<int32_t> &point_nodes);

}  // namespace dl
