// Output modules of a run: the reference's GroupOutputModule,
// SampleModule, CSVOutputModule (CSVDataPrinter) and ParaViewModule, written
// from the host after the steps their conditions select.  The writers read
// the engine through OutputHost, so they see the engine's public state only.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dynlattice.h"
#include "pro.hpp"

namespace dl {

// What the output modules read from an engine (original node/element numbering).
class OutputHost {
 public:
  virtual ~OutputHost() = default;
  virtual int n_nodes() = 0;
  virtual int n_elems() = 0;
  virtual int nodes_per_elem() = 0;                         // 2, 3 or 4
  virtual void reference_coords(double *X0) = 0;           // [N][3]
  virtual void connectivity(int32_t *conn) = 0;             // [E][nodes_per_elem], along the line
  virtual void state(double *u, double *th, double *v) = 0;  // [N][3], [N][3], [N][6]
  virtual void internal_force(const double *u, const double *th, double *f) = 0;  // [N][6]
  virtual void external_force(double *f) = 0;               // [N][6] at the current time
  // element table of GET_TABLE ("strain", "stress", "mat_strain", "mat_stress",
  // "plast_strain") at the current state, [E][6]
  virtual void element_table(const std::string &name, double *out) = 0;
  virtual void energies(dl_energies *e) = 0;
  virtual void time(double *t, double *dt, int64_t *step) = 0;
  virtual void run(int64_t nsteps) = 0;
  virtual bool adaptive() = 0;  // time step decided on the device (MilneDevice)
};

// VTU point data beyond displacements, velocities and rotations
enum { VTU_FINT = 1, VTU_FEXT = 2, VTU_FRES = 4 };

// One ParaView UnstructuredGrid piece of the whole mesh at the current state
// (ParaViewModule::writeFile_/writePiece_, ParaViewModule.cpp:236-620), with
// the named element tables as cell data (el_data, :579-618).
void write_vtu(OutputHost &h, const std::string &path, int node_data,
               const std::vector<std::string> &el_data = {});

// ParaView collection file (ParaViewModule::run, ParaViewModule.cpp:182-216).
void write_pvd(const std::string &path, const std::vector<double> &times, const std::vector<std::string> &files);

// Run a parsed .pro file's control loop on an engine with its output
// modules, until control.runWhile ends or max_steps steps (< 0: no cap).
// Output paths are taken relative to out_dir.  Returns the steps run.
int64_t run_pro(OutputHost &h, const ProModel &M, const std::string &out_dir, int64_t max_steps);

}  // namespace dl
