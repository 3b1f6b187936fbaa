// opt_heat_gpu.cpp -- ICARAT's opt-heat app (opt-heat/opt_heat.cpp:12-151) on
// the B200 library: LinearHeat on a quad4 / hexa8 box, Helmholtz (PDE)
// density filter, threshold projection, Jacobi-PCG heat solve, objective
// u^T K u, volume constraint sum x v - V0, MMA.  The loop runs on the device
// (icb_run_heat) with the app's stop rule, Optimize::isConvergence(1e-7, 50)
// and at most 1000 steps; every step appends to function.csv and writes
// res<step>.vtk (temperature, threshold_s, design_s) as the app does, in the
// legacy-VTK text of export_vtk.hpp (the app's meshio binary conversion is
// not run).  One line per step on stdout: "step,objective".
//
// usage: opt_heat_gpu <config.toml>
// [this_problem] keys: filterR (the app's filter radius); optional steps
// (fixed count instead of the stop rule), vtk (false: no res<step>.vtk).
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "icarat_export.hpp"
#include "icarat_gpu.hpp"

using namespace icarat;

namespace
{
template <class T> T option(const toml::value &cfg, const char *key, T dflt)
{
  if(!cfg.contains("this_problem") || !cfg.at("this_problem").contains(key))
    return dflt;
  return toml::get<T>(cfg.at("this_problem").at(key));
}

/// range rows [[x0, x1], [y0, y1], [z0, z1]] -> {x0, x1, y0, y1, z0, z1}
void box(const toml::value &rows, double r[6])
{
  const toml::array &a = rows.as_array();
  for(int k = 0; k < 3; k++)
  {
    const toml::array &p = a.at(k).as_array();
    r[2 * k] = p.at(0).as_floating();
    r[2 * k + 1] = p.at(1).as_floating();
  }
}

struct Run
{
  int dim;
  std::vector<Node> node;
  std::vector<Element> element;
  bool vtk;
};

/// output() of opt_heat.cpp:194-246 and the addPlot of the step
void on_step(void *user, int step, double f, const double *rho, const double *temp, const double *)
{
  Run &R = *static_cast<Run *>(user);
  std::printf("%d,%.17g\n", step, f);
  addPlot(step, f, "function.csv", step);
  if(!R.vtk)
    return;
  std::ofstream fout("res" + std::to_string(step) + ".vtk");
  makeHeaderVTK(fout);
  setPointVTK(R.node, fout);
  setElementVTK(R.element, fout);
  setElementTypeVTK(R.dim, R.element, fout);
  addPointScalarVTK("temperature", R.node, fout, true, [&](Node &n) { return temp[n.ID]; });
  std::vector<double> nd(R.node.size(), 0.0);
  for(const Element &e : R.element)
    for(int id : e.nodeID)
      nd[id] += rho[e.ID] / e.ne;
  addPointScalarVTK("threshold_s", R.node, fout, false,
                    [&](Node &n) { return nd[n.ID] > 0.5 ? 1.0 : 0.0; });
  addElementScalarVTK("design_s", R.element, fout, true, [&](Element &e) { return rho[e.ID]; });
}
} // namespace

int main(int argc, char **argv)
{
  if(argc != 2)
  {
    std::fprintf(stderr, "usage: %s <.toml file>\n", argv[0]);
    return 1;
  }
  const toml::value config = toml::parse(argv[1]);
  const double filterR = toml::find<double>(config, "this_problem", "filterR");
  const int fixedSteps = option<int>(config, "steps", 0);

  // [mesh] (MeshIcarat::setParameter("heat"))
  const toml::value &mesh = toml::find(config, "mesh");
  const int dim = toml::find<int>(mesh, "dimension");
  const std::string type = toml::find<std::string>(mesh, "type");
  if(!((type == "quad4" && dim == 2) || (type == "hexa8" && dim == 3)))
  {
    std::fprintf(stderr, "Error: mesh type \"%s\" is not available (quad4 in 2D, hexa8 in 3D)\n",
                 type.c_str());
    return 1;
  }
  const auto div = toml::find<std::array<int, 3>>(mesh, "division");
  const auto len = toml::find<std::array<double, 3>>(mesh, "length");

  // [material] (Heat::setParameter, heat.cpp:18-64)
  const toml::value &mat = toml::find(config, "material");
  if(toml::find<std::string>(mat, "type") != "Heat")
  {
    std::fprintf(stderr, "Error: [material] type must be \"Heat\"\n");
    return 1;
  }
  icb_heat_desc hd{};
  hd.dim = dim;
  hd.nx = div[0];
  hd.ny = div[1];
  hd.nz = dim == 3 ? div[2] : 1;
  hd.lx = len[0];
  hd.ly = len[1];
  hd.lz = dim == 3 ? len[2] : 1.0;
  const toml::array &cond = toml::find(mat, "conductivity").as_array();
  for(int k = 0; k < 6; k++)
  {
    hd.cond1[k] = cond.at(0).as_array().at(k).as_floating();
    hd.cond2[k] = cond.at(1).as_array().at(k).as_floating();
  }
  hd.penalty = toml::find<double>(mat, "penalty");
  const double design0 = toml::find<double>(mat, "designs_0");

  icb_heat h = nullptr;
  check(icb_heat_create(detail::shared_context(), &hd, &h), "icb_heat_create");

  // [boundary_condition] with one DOF per node (input_dirich / input_neumann)
  const toml::value &bc = toml::find(config, "boundary_condition");
  if(bc.contains("dirichlet"))
    for(const toml::value &row : bc.at("dirichlet").as_array())
    {
      const toml::array &r = row.as_array();
      double range[6];
      box(r.at(2), range);
      check(icb_heat_dirichlet_box(h, int(r.at(0).as_array().at(0).as_integer()),
                                   r.at(1).as_array().at(0).as_floating(), range),
            "icb_heat_dirichlet_box");
    }
  if(bc.contains("neumann"))
    for(const toml::value &row : bc.at("neumann").as_array())
    {
      const toml::array &r = row.as_array();
      double range[6];
      box(r.at(1), range);
      check(icb_heat_flux_box(h, r.at(0).as_array().at(0).as_floating(), range),
            "icb_heat_flux_box");
    }
  long long numeq = 0;
  check(icb_heat_finalize(h, &numeq), "icb_heat_finalize");

  // nodes and elements of the box (meshBox order) for the VTK files
  Run R;
  R.dim = dim;
  R.vtk = option<bool>(config, "vtk", true);
  const long long nx = div[0], ny = div[1], nz = dim == 3 ? div[2] : 1;
  const long long sx = nx + 1, sxy = sx * (ny + 1), nnode = sxy * (dim == 3 ? nz + 1 : 1);
  const long long nel = nx * ny * nz;
  R.node.resize(nnode);
  for(long long n = 0; n < nnode; n++)
  {
    Node &q = R.node[n];
    q.ID = int(n);
    q.x[0] = len[0] / double(nx) * double(n % sx);
    q.x[1] = len[1] / double(ny) * double((n / sx) % (ny + 1));
    q.x[2] = dim == 3 ? len[2] / double(nz) * double(n / sxy) : 0.0;
  }
  R.element.resize(nel);
  for(long long e = 0; e < nel; e++)
  {
    Element &el = R.element[e];
    el.ID = int(e);
    el.ne = dim == 2 ? 4 : 8;
    const long long i = e % nx, j = (e / nx) % ny, k = e / (nx * ny);
    const long long b = i + j * sx + (dim == 3 ? k * sxy : 0);
    const long long nd[4] = {b, b + 1, b + 1 + sx, b + sx};
    for(long long v : nd)
      el.nodeID.push_back(int(v));
    if(dim == 3)
      for(long long v : nd)
        el.nodeID.push_back(int(v + sxy));
  }

  // the loop (opt_heat.cpp:79-151): at most 1000 steps, isConvergence(1e-7, 50)
  const int maxSteps = fixedSteps > 0 ? fixedSteps : 1000;
  icb_loop_opts o{};
  o.nsteps = maxSteps;
  o.filter_radius = filterR;
  o.solve.precision = ICB_FP64;
  o.solve.precond = ICB_PRECOND_JACOBI;
  o.solve.tol = 1e-10;
  o.solve.maxit = 10000;
  o.on_step = on_step;
  o.step_user = &R;
  o.conv_eps = fixedSteps > 0 ? 0.0 : 1.0e-7;
  o.conv_min_steps = 50;
  int done = 0;
  o.steps_done = &done;
  std::vector<double> rho0(nel, design0), hist(maxSteps), x(nel);
  check(icb_run_heat(h, &o, rho0.data(), hist.data(), x.data()), "icb_run_heat");
  if(fixedSteps == 0 && done == maxSteps)
    std::fprintf(stderr, "not convergence in this optimization\n");
  icb_heat_destroy(h);
  return 0;
}
