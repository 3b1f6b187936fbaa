// opt_mma_helmholtz_gpu.cpp -- ICARAT's opt-mma-HelmholtzFilter app
// (opt-mma-HelmholtzFilter/opt_mma_Helmholtz.cpp:12-163) written against the
// B200 shim: Helmholtz (PDE) density filter, threshold projection, linear
// analysis, sensitivities scaled by 1/V0, MMA update with the volume
// constraint sum x v / V0 - 1.  No VTK / CSV / FDM output; one line per step
// on stdout: "step,compliance,constraint".
//
// usage: opt_mma_helmholtz_gpu <config.toml>
// [this_problem] keys (all optional): steps (fixed count; default: the app's
// isConvergence(1e-7, 50) rule, at most 1000 steps), filter_radius
// (default 2 x the element size, as the app), volume_ref (V0; default the
// step-1 volume), solver ("Eigen_LDLT").
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
  const std::string solver = option<std::string>(config, "solver", "Eigen_LDLT");
  double V0 = option<double>(config, "volume_ref", 0.0);

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
  MMASolver mma(fem.nelx, 1);
  const double radius =
      option<double>(config, "filter_radius", 2.0 * std::fabs(node[0].x[0] - node[1].x[0]));
  FilterHelmholtz<LinearElastic, Node> filter(fem, element, node, radius);
  for(int i = 0; i < fem.nelx; i++)
    optim.design_s[i] = element[i].design_s();
  LinearAnalysis<LinearElastic, Node> compt(fem, element, node, force, dis);

  std::vector<double> dv;
  for(int running = 1; running;)
  {
    optim.optstep++;
    std::vector<double> xf = filter.densityFilter(optim.design_s, "Eigen_CG", 0, false);
    const double beta = std::min(std::pow(2.0, optim.optstep / 40), 16.0);
    std::vector<double> xh = filter.threshold(xf, beta, 0.5);
    for(int i = 0; i < fem.nelx; i++)
      element[i].setDesignS(xh[i]);

    compt.solve(solver, false);

    double vol = 0.0;
    for(int i = 0; i < fem.nelx; i++)
      vol += element[i].design_s() * element[i].volume;
    if(optim.optstep == 1 && V0 <= 0.0)
    {
      V0 = vol;
      optim.const_h[0] = 0.0;
    }
    else
      optim.const_h[0] = vol / V0 - 1.0;
    optim.object_f = dis.val.dot(force.fext);
    std::printf("%d,%.17g,%.17g\n", optim.optstep, optim.object_f, optim.const_h[0]);

    running = fixedSteps > 0 ? optim.optstep < fixedSteps
                             : (optim.isConvergence(1.0e-7, 50) && optim.optstep < 1000);
    if(!running)
      break;

    sensitivity(fem, optim.dfds, &dv);
    std::vector<double> dxh = filter.thresholdDerivative(xf, beta, 0.5);
    for(int i = 0; i < fem.nelx; i++)
    {
      optim.dfds[i] *= dxh[i];
      optim.dgds[i] = dv[i] / V0 * dxh[i];
    }
    optim.dfds = filter.densityFilter(optim.dfds, "Eigen_CG", 0, true);
    optim.dgds = filter.densityFilter(optim.dgds, "Eigen_CG", 0, true);
    mma.Update(optim.design_s.data(), optim.dfds.data(), optim.const_h.data(), optim.dgds.data(),
               optim.xmin.data(), optim.xmax.data());
  }
  return 0;
}
