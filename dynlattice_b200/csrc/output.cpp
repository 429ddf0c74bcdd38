// Output modules of a .pro run: see output.hpp.
#include "output.hpp"

#include <zlib.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <memory>
#include <stdexcept>

#include "expr.hpp"

namespace dl {

namespace {

// a text file, gzip-compressed when its name ends in ".gz" (the reference's
// Sample and CSVOutput files, e.g. "$(CASE_NAME)/disp.gz")
class TextOut {
 public:
  explicit TextOut(const std::string &path) {
    const std::filesystem::path p(path);
    if (p.has_parent_path()) std::filesystem::create_directories(p.parent_path());
    gz_ = path.size() > 3 && path.compare(path.size() - 3, 3, ".gz") == 0;
    if (gz_) {
      z_ = gzopen(path.c_str(), "wb");
      if (!z_) throw std::runtime_error("cannot open " + path);
    } else {
      f_ = std::fopen(path.c_str(), "w");
      if (!f_) throw std::runtime_error("cannot open " + path);
    }
  }
  ~TextOut() {
    if (z_) gzclose(z_);
    if (f_) std::fclose(f_);
  }
  TextOut(const TextOut &) = delete;
  TextOut &operator=(const TextOut &) = delete;
  void put(const std::string &s) {
    if (gz_) {
      if (!s.empty() && gzwrite(z_, s.data(), static_cast<unsigned>(s.size())) == 0)
        throw std::runtime_error("gzip write failed");
    } else if (std::fwrite(s.data(), 1, s.size(), f_) != s.size()) {
      throw std::runtime_error("write failed");
    }
  }

 private:
  bool gz_ = false;
  gzFile z_ = nullptr;
  std::FILE *f_ = nullptr;
};

std::string num(double x) {
  char b[32];
  std::snprintf(b, sizeof b, "%.17g", x);
  return b;
}

// values of a ParaView DataArray: single precision, as ParaView reads them
// (ParaViewModule::writeDataArray_, :627-648)
void data_array(std::string &o, const char *name, int comps, int rows, const double *v, int stride, int off) {
  o += "      <DataArray type=\"Float32\" Name=\"";
  o += name;
  o += "\" NumberOfComponents=\"" + std::to_string(comps) + "\">\n";
  char b[32];
  for (int r = 0; r < rows; ++r) {
    o += "        ";
    for (int c = 0; c < comps; ++c) {
      std::snprintf(b, sizeof b, "%.8e ", static_cast<double>(static_cast<float>(v[r * stride + off + c])));
      o += b;
    }
    o += "\n";
  }
  o += "      </DataArray>\n";
}

}  // namespace

void write_vtu(OutputHost &h, const std::string &path, int node_data, const std::vector<std::string> &el_data) {
  const int N = h.n_nodes(), E = h.n_elems();
  std::vector<double> X0(static_cast<size_t>(N) * 3), u(X0.size()), th(X0.size()), v(static_cast<size_t>(N) * 6);
  const int nen = h.nodes_per_elem();
  std::vector<int32_t> conn(static_cast<size_t>(E) * nen);
  h.reference_coords(X0.data());
  h.connectivity(conn.data());
  h.state(u.data(), th.data(), v.data());
  std::string o;
  o.reserve(static_cast<size_t>(N) * 200 + static_cast<size_t>(E) * 40);
  o += "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\">\n  <UnstructuredGrid>\n";
  o += "    <Piece NumberOfPoints=\"" + std::to_string(N) + "\" NumberOfCells=\"" + std::to_string(E) + "\">\n";
  // points: the reference coordinates (ParaView warps them by "Displacement")
  o += "    <Points>\n      <DataArray type=\"Float32\" NumberOfComponents=\"3\">\n";
  char b[96];
  for (int n = 0; n < N; ++n) {
    std::snprintf(b, sizeof b, "        %.8e %.8e %.8e\n", X0[n * 3], X0[n * 3 + 1], X0[n * 3 + 2]);
    o += b;
  }
  o += "      </DataArray>\n    </Points>\n    <Cells>\n";
  o += "      <DataArray type=\"Int32\" Name=\"connectivity\">\n";
  // VTK's node order of a higher-order line: the two ends, then the interior
  // nodes (ParaViewModule::gmsh2ParaNodeOrder, ParaViewModule.cpp:788-830)
  static const int vorder[5][4] = {{0}, {0}, {0, 1}, {0, 2, 1}, {0, 3, 1, 2}};
  for (int e = 0; e < E; ++e) {
    o += "       ";
    for (int a = 0; a < nen; ++a) o += " " + std::to_string(conn[static_cast<size_t>(e) * nen + vorder[nen][a]]);
    o += "\n";
  }
  o += "      </DataArray>\n      <DataArray type=\"Int32\" Name=\"offsets\">\n";
  for (int e = 0; e < E; ++e) o += "        " + std::to_string(nen * (e + 1)) + "\n";
  o += "      </DataArray>\n      <DataArray type=\"UInt8\" Name=\"types\">\n";
  // VTK_LINE, VTK_QUADRATIC_EDGE, VTK_CUBIC_LINE (ParaViewModule::nameToVTKNum, :712-731)
  const char *vtype = nen == 2 ? "3" : (nen == 3 ? "21" : "35");
  for (int e = 0; e < E; ++e) o += std::string("        ") + vtype + "\n";
  o += "      </DataArray>\n    </Cells>\n";
  o += "    <PointData Vectors=\"Displacement\">\n";
  data_array(o, "Displacement", 3, N, u.data(), 3, 0);
  data_array(o, "Velocity", 3, N, v.data(), 6, 0);
  data_array(o, "otherDofsDisp", 3, N, th.data(), 3, 0);
  data_array(o, "otherDofsVelo", 3, N, v.data(), 6, 3);
  if (node_data & (VTU_FINT | VTU_FEXT | VTU_FRES)) {
    std::vector<double> fi(static_cast<size_t>(N) * 6, 0.0), fe(fi.size(), 0.0), fr(fi.size());
    if (node_data & (VTU_FINT | VTU_FRES)) h.internal_force(u.data(), th.data(), fi.data());
    if (node_data & (VTU_FEXT | VTU_FRES)) h.external_force(fe.data());
    for (size_t k = 0; k < fr.size(); ++k) fr[k] = fe[k] - fi[k];
    if (node_data & VTU_FINT) {
      data_array(o, "Internal Forces", 3, N, fi.data(), 6, 0);
      data_array(o, "Internal Torques", 3, N, fi.data(), 6, 3);
    }
    if (node_data & VTU_FEXT) {
      data_array(o, "External Forces", 3, N, fe.data(), 6, 0);
      data_array(o, "External Torques", 3, N, fe.data(), 6, 3);
    }
    if (node_data & VTU_FRES) {
      data_array(o, "Resulting Forces", 3, N, fr.data(), 6, 0);
      data_array(o, "Resulting Torques", 3, N, fr.data(), 6, 3);
    }
  }
  o += "    </PointData>\n    <CellData>\n";
  if (!el_data.empty()) {
    std::vector<double> tab(static_cast<size_t>(E) * 6);
    for (const std::string &name : el_data) {
      h.element_table(name, tab.data());
      data_array(o, name.c_str(), 6, E, tab.data(), 6, 0);
    }
  }
  o += "    </CellData>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>";
  TextOut f(path);
  f.put(o);
}

void write_pvd(const std::string &path, const std::vector<double> &times, const std::vector<std::string> &files) {
  if (times.size() != files.size()) throw std::invalid_argument("pvd: one time per file");
  std::string o = "<?xml version=\"1.0\"?>\n<VTKFile type=\"Collection\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
  o += "  <Collection>\n";
  for (size_t i = 0; i < files.size(); ++i)
    o += "    <DataSet timestep=\"" + num(times[i]) + "\" group=\"\" part=\"0\" file=\"" + files[i] + "\" />\n";
  o += "  </Collection>\n</VTKFile>\n";
  TextOut f(path);
  f.put(o);
}

namespace {

// The variables output expressions may use: time, step, time step, run time,
// the energies and the GroupOutput variables <group>.<load|resp|disp|velo>.<dof>.
struct OutVars {
  std::vector<std::string> names;
  std::vector<double> vals;
  int add(const std::string &n) {
    names.push_back(n);
    vals.push_back(0.0);
    return static_cast<int>(names.size()) - 1;
  }
};

struct GroupVar {
  std::vector<int32_t> nodes;
  int dof;
  int i_load, i_resp, i_disp, i_velo;
};

struct Module {
  const ProOutput *o;
  ExprPtr when;      // null: every step
  bool time_only = false;
  std::vector<ExprPtr> data;  // Sample dataSets
  std::unique_ptr<TextOut> file;
  bool header = false;
  int count = 0;     // ParaView files written
  std::vector<double> pvd_t;
  std::vector<std::string> pvd_f;
};

}  // namespace

int64_t run_pro(OutputHost &h, const ProModel &M, const std::string &out_dir, int64_t max_steps) {
  const int N = h.n_nodes();
  auto out_path = [&](const std::string &p) {
    return (out_dir.empty() || p.empty() || p[0] == '/') ? p : out_dir + "/" + p;
  };
  OutVars V;
  const int i_t = V.add("t"), i_i = V.add("i"), i_dt = V.add("deltaTime"), i_run = V.add("runtime");
  const int i_ek = V.add("kineticEnergy"), i_ep = V.add("potentialEnergy"), i_ed = V.add("dissipatedEnergy");
  const int i_wx = V.add("externalWork");
  std::vector<GroupVar> gvars;
  for (const ProOutput &o : M.outputs) {
    if (o.type != "GroupOutput") continue;
    for (const std::string &g : o.node_groups) {
      auto it = M.groups.find(g);
      if (it == M.groups.end()) throw std::runtime_error("GroupOutput: no node group " + g);
      for (const std::string &d : o.dofs) {
        int dof = -1;
        for (size_t k = 0; k < M.dof_names.size(); ++k)
          if (M.dof_names[k] == d) dof = static_cast<int>(k);
        if (dof < 0) throw std::runtime_error("GroupOutput: unknown DOF " + d);
        GroupVar gv{it->second, dof, V.add(g + ".load." + d), V.add(g + ".resp." + d), V.add(g + ".disp." + d),
                    V.add(g + ".velo." + d)};
        gvars.push_back(gv);
      }
    }
  }
  const std::vector<std::string> tnames = {"t", "i", "deltaTime"};
  std::vector<Module> mods;
  for (const ProOutput &o : M.outputs) {
    if (o.type == "GroupOutput") continue;
    Module md;
    md.o = &o;
    if (!o.when.empty()) {
      md.when = parseExpr(o.when, V.names);
      try {
        parseExpr(o.when, tnames);
        md.time_only = true;
      } catch (const std::exception &) {
        md.time_only = false;
      }
    } else {
      md.time_only = true;
    }
    if (o.type == "Sample") {
      for (const std::string &d : o.data_sets) md.data.push_back(parseExpr(d, V.names));
      md.file = std::make_unique<TextOut>(out_path(o.file));
    } else if (o.type == "CSVOutput") {
      md.file = std::make_unique<TextOut>(out_path(o.file));
    }
    mods.push_back(std::move(md));
  }
  auto fires = [&](const Module &md, const double *vars) {
    return !md.when || evalExpr(md.when.get(), vars) != 0.0;
  };
  bool all_time_only = true;
  for (const Module &md : mods) all_time_only = all_time_only && md.time_only;
  const auto wall0 = std::chrono::steady_clock::now();
  std::vector<double> u(static_cast<size_t>(N) * 3), th(u.size()), v(static_cast<size_t>(N) * 6),
      fi(static_cast<size_t>(N) * 6), fe(fi.size());
  // all variables at the current state
  auto refresh = [&](double t, double dt, int64_t step) {
    V.vals[i_t] = t;
    V.vals[i_i] = static_cast<double>(step);
    V.vals[i_dt] = dt;
    V.vals[i_run] = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
    dl_energies e{};
    h.energies(&e);
    V.vals[i_ek] = e.kinetic;
    V.vals[i_ep] = e.potential;
    V.vals[i_ed] = e.dissipated;
    V.vals[i_wx] = e.external_work;
    h.state(u.data(), th.data(), v.data());
    if (!gvars.empty()) {
      h.internal_force(u.data(), th.data(), fi.data());
      h.external_force(fe.data());
      // GroupOutputModule::run (GroupOutputModule.cpp:121-150): sums of load
      // and response, means of displacement and velocity
      for (const GroupVar &g : gvars) {
        double sl = 0, sr = 0, sd = 0, sv = 0;
        for (int32_t n : g.nodes) {
          sl += fe[static_cast<size_t>(n) * 6 + g.dof];
          sr += fi[static_cast<size_t>(n) * 6 + g.dof];
          sd += g.dof < 3 ? u[static_cast<size_t>(n) * 3 + g.dof] : th[static_cast<size_t>(n) * 3 + g.dof - 3];
          sv += v[static_cast<size_t>(n) * 6 + g.dof];
        }
        const double cnt = std::max<size_t>(1, g.nodes.size());
        V.vals[g.i_load] = sl;
        V.vals[g.i_resp] = sr;
        V.vals[g.i_disp] = sd / cnt;
        V.vals[g.i_velo] = sv / cnt;
      }
    }
  };
  auto write_outputs = [&](double t) {
    for (Module &md : mods) {
      if (!fires(md, V.vals.data())) continue;
      const ProOutput &o = *md.o;
      if (o.type == "Sample") {
        std::string row;
        for (size_t k = 0; k < md.data.size(); ++k) {
          if (k) row += o.separator;
          row += num(evalExpr(md.data[k].get(), V.vals.data()));
        }
        md.file->put(row + "\n");
      } else if (o.type == "CSVOutput") {
        // CSVDataPrinter: a header "time,label,<dof>[<node>]..." then one row
        // "t,label,values..." per vector (CSVDataPrinter.cpp:84-227)
        if (!md.header) {
          std::string hd = "time,label";
          for (int n = 0; n < N; ++n)
            for (const std::string &d : M.dof_names) hd += "," + d + "[" + std::to_string(n) + "]";
          md.file->put(hd + "\n");
          md.header = true;
        }
        for (const std::string &vs : o.vectors) {
          const size_t eq = vs.find('=');
          auto trim = [](std::string s) {
            s.erase(0, s.find_first_not_of(" \t"));
            s.erase(s.find_last_not_of(" \t") + 1);
            return s;
          };
          // "<vector> = <label>" (CSVOutput.vectors: "state = disp" prints the state as "disp")
          const std::string vec = trim(eq == std::string::npos ? vs : vs.substr(0, eq));
          const std::string label = trim(eq == std::string::npos ? vs : vs.substr(eq + 1));
          std::string row = num(t) + "," + label;
          for (int n = 0; n < N; ++n)
            for (int k = 0; k < 6; ++k) {
              double x;
              if (vec == "state" || vec == "disp") x = k < 3 ? u[n * 3 + k] : th[n * 3 + k - 3];
              else if (vec == "state1" || vec == "velo") x = v[n * 6 + k];
              else throw std::runtime_error("CSVOutput: unknown vector " + vec);
              row += "," + num(x);
            }
          md.file->put(row + "\n");
        }
      } else if (o.type == "ParaView") {
        const size_t pos = o.format.rfind("%i");
        std::string name = o.format;
        if (pos != std::string::npos) name.replace(pos, 2, std::to_string(md.count));
        ++md.count;
        int nd = 0;
        for (const std::string &d : o.node_data) {
          if (d == "fint") nd |= VTU_FINT;
          else if (d == "fext") nd |= VTU_FEXT;
          else if (d == "fres") nd |= VTU_FRES;
        }
        const std::string file = name + ".vtu";
        write_vtu(h, out_path(file), nd, o.el_data);
        if (pos != std::string::npos) {
          md.pvd_t.push_back(t);
          md.pvd_f.push_back(std::filesystem::path(file).filename().string());
          const std::string pvd = o.format.substr(0, pos) + o.format.substr(pos + 2) + ".pvd";
          write_pvd(out_path(pvd), md.pvd_t, md.pvd_f);
        }
      }
    }
  };
  double t = 0, dt = 0;
  int64_t step = 0;
  h.time(&t, &dt, &step);
  const int64_t step0 = step;
  const double t_end = M.t_end;
  auto more = [&](double tt, int64_t st) {
    if (max_steps >= 0 && st - step0 >= max_steps) return false;
    if (t_end >= 0.0) return tt < t_end * (1.0 - 1e-12);
    return M.steps < 0 || st < M.steps;
  };
  while (more(t, step)) {
    int64_t k = 1;
    if (!h.adaptive() && all_time_only) {
      // fixed dt: run up to the next step at which a module fires or the run ends
      double tk = t;
      double tv[3];
      for (;; ++k) {
        tk += dt;
        tv[0] = tk;
        tv[1] = static_cast<double>(step + k);
        tv[2] = dt;
        if (!more(tk, step + k)) break;
        bool any = false;
        for (const Module &md : mods) any = any || !md.when || evalExpr(md.when.get(), tv) != 0.0;
        if (any) break;
      }
    }
    h.run(k);
    h.time(&t, &dt, &step);
    if (mods.empty()) continue;
    refresh(t, dt, step);
    write_outputs(t);
  }
  return step - step0;
}

}  // namespace dl
