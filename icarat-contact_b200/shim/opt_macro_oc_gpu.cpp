// opt_macro_oc_gpu.cpp -- ICARAT's opt-macro-oc app (opt-macro-oc/opt_macro_oc.cpp:
// 13-172) written against the B200 shim: cone density filter, threshold
// projection, linear analysis, sensitivities, OC update with the filtered and
// thresholded volume constraint.  No VTK / CSV output; one line per step on
// stdout: "step,compliance,volume".
//
// usage: opt_macro_oc_gpu <config.toml>
// [this_problem] keys (all optional): steps (fixed step count; default: the
// app's stopping rule isConvergence(1e-7, 50), at most 1000 steps),
// filter_radius (3.0), move_limit (0.15), solver ("Eigen_CG"), threshold (true).
#include <algorithm>
#include <cstdio>

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
} // namespace

int main(int argc, char **argv)
{
  if(argc != 2)
  {
    std::fprintf(stderr, "usage: %s <.toml file>\n", argv[0]);
    return 1;
  }
  const toml::value config = toml::parse(argv[1]);
  const int fixedSteps = option<int>(config, "steps", 0);
  const double radius = option<double>(config, "filter_radius", 3.0);
  const double move = option<double>(config, "move_limit", 0.15);
  const std::string solver = option<std::string>(config, "solver", "Eigen_CG");
  const bool useThreshold = option<bool>(config, "threshold", true);
  const double T = 0.5;

  FEM fem;
  MeshIcarat<LinearElastic, Node> mesh(fem, config);
  mesh.setParameter("structure");
  std::vector<LinearElastic> element;
  for(int type = 0; type < mesh.numeleTypes(); type++)
    for(int e = 0; e < mesh.nelx(type); e++)
    {
      LinearElastic el(fem.voigt, mesh.ne(type), mesh.ipmax(type), mesh.ne(type) * fem.dofnp);
      el.setParameter(config);
      element.push_back(el);
    }
  std::vector<Node> node(fem.numnp);
  mesh.generate(element, node);

  BCIcarat<LinearElastic, Node> BC(fem, element, node);
  BC.input_dirich(config);
  fem.numeq = BC.makeDOF();
  Force force(fem.numeq);
  Value dis(fem.numeq);
  BC.input_neumann(config, force);

  Optimize optim(fem.nelx, 1, 1.0e-4, 1.0);
  OC oc(fem.nelx);
  oc.setMoveLimit(move);
  Filter<LinearElastic, Node> filter(fem, element, node, radius);
  for(int i = 0; i < fem.nelx; i++)
    optim.design_s[i] = element[i].design_s();
  LinearAnalysis<LinearElastic, Node> compt(fem, element, node, force, dis);

  double V0 = 0.0;
  std::vector<double> dv;
  for(int running = 1; running;)
  {
    optim.optstep++;
    std::vector<double> xf = filter.densityFilter(optim.design_s, false);
    const double beta = useThreshold ? std::min(std::pow(2.0, optim.optstep / 40), 16.0) : 0.0;
    std::vector<double> xh = beta > 0.0 ? filter.threshold(xf, beta, T) : xf;
    std::vector<double> dxh = beta > 0.0 ? filter.thresholdDerivative(xf, beta, T)
                                         : std::vector<double>(xf.size(), 1.0);
    for(int i = 0; i < fem.nelx; i++)
      element[i].setDesignS(xh[i]);

    compt.solve(solver, false);
    optim.object_f = dis.val.dot(force.fext);

    double vol = 0.0;
    for(int i = 0; i < fem.nelx; i++)
      vol += element[i].design_s() * element[i].volume;
    if(optim.optstep == 1)
      V0 = vol;
    std::printf("%d,%.17g,%.17g\n", optim.optstep, optim.object_f, vol);

    running = fixedSteps > 0 ? optim.optstep < fixedSteps
                             : (optim.isConvergence(1.0e-7, 50) && optim.optstep < 1000);
    if(!running)
      break;

    sensitivity(fem, optim.dfds, &dv);
    for(int i = 0; i < fem.nelx; i++)
    {
      optim.dfds[i] *= dxh[i];
      optim.dgds[i] = dv[i] * dxh[i];
    }
    optim.dfds = filter.densityFilter(optim.dfds, true);
    optim.dgds = filter.densityFilter(optim.dgds, true);
    oc.UpdateVariables(optim.design_s, optim.dfds, V0, optim.dgds, optim.xmin, optim.xmax,
                       oc_volume(fem, filter, beta, T));
  }
  return 0;
}
