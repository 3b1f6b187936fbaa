// opt_macro_gcmma_gpu.cpp -- ICARAT's opt-macro-gcmma app (opt_macro_gcmma.cpp:
// 12-238) on the B200 shim: cone filter of radius 2 h, threshold with
// beta = min(int(max((step - 100) / 40, 1)), 8), linear analysis, constraint
// sum x v - V0, sensitivities (dv = v) times the threshold derivative, adjoint
// filter, GCMMA outer update, evaluation of the candidate and up to 15 inner
// updates until the approximation is conservative.  One line per step on
// stdout: "step,compliance,constraint,inner iterations".
//
// usage: opt_macro_gcmma_gpu <config.toml>
// [this_problem] keys (all optional): steps (fixed count; default the app's
// isConvergence(1e-7, 50) rule, at most 1000 steps), solver ("Eigen_CG").
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
  const std::string solver = option<std::string>(config, "solver", "Eigen_CG");
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
  GCMMASolver gcmma(fem.nelx, 1);
  const double filterR = 2.0 * mesh.length()[0] / mesh.div()[0];
  Filter<LinearElastic, Node> filter(fem, element, node, filterR);
  for(int i = 0; i < fem.nelx; i++)
    optim.design_s[i] = element[i].design_s();
  LinearAnalysis<LinearElastic, Node> compt(fem, element, node, force, dis);

  double V0 = 0.0;
  std::vector<double> dv, xnew(fem.nelx);
  // filter, threshold and solve at x: compliance and volume sum_e x v
  auto evaluate = [&](const std::vector<double> &x, double beta, double &f, double &vol,
                      std::vector<double> *dxh) {
    std::vector<double> xf = filter.densityFilter(x, false);
    std::vector<double> xh = filter.threshold(xf, beta, T);
    if(dxh)
      *dxh = filter.thresholdDerivative(xf, beta, T);
    for(int i = 0; i < fem.nelx; i++)
      element[i].setDesignS(xh[i]);
    compt.solve(solver, false);
    f = dis.val.dot(force.fext);
    vol = 0.0;
    for(int i = 0; i < fem.nelx; i++)
      vol += element[i].design_s() * element[i].volume;
  };
  for(int running = 1; running;)
  {
    optim.optstep++;
    const int btmp = int(std::max((optim.optstep - 100) / 40.0, 1.0));
    const double beta = std::min(double(btmp), 8.0);
    std::vector<double> dxh;
    double vol;
    evaluate(optim.design_s, beta, optim.object_f, vol, &dxh);
    if(optim.optstep == 1)
      V0 = vol;
    optim.const_h[0] = vol - V0;

    const bool last = fixedSteps > 0 ? optim.optstep >= fixedSteps
                                     : !(optim.isConvergence(1.0e-7, 50) && optim.optstep < 1000);
    sensitivity(fem, optim.dfds, &dv);
    for(int i = 0; i < fem.nelx; i++)
    {
      optim.dfds[i] *= dxh[i];
      optim.dgds[i] = dv[i] * dxh[i];
    }
    optim.dfds = filter.densityFilter(optim.dfds, true);
    optim.dgds = filter.densityFilter(optim.dgds, true);

    gcmma.OuterUpdate(xnew.data(), optim.design_s.data(), optim.object_f, optim.dfds.data(),
                      optim.const_h.data(), optim.dgds.data(), optim.xmin.data(),
                      optim.xmax.data());
    double fnew, vnew;
    evaluate(xnew, beta, fnew, vnew, nullptr);
    double hnew = vnew - V0;
    int k = 0;
    for(; !gcmma.ConCheck(fnew, &hnew) && k < 15; k++)
    {
      gcmma.InnerUpdate(xnew.data(), fnew, &hnew, optim.design_s.data(), optim.object_f,
                        optim.dfds.data(), optim.const_h.data(), optim.dgds.data(),
                        optim.xmin.data(), optim.xmax.data());
      evaluate(xnew, beta, fnew, vnew, nullptr);
      hnew = vnew - V0;
    }
    std::printf("%d,%.17g,%.17g,%d\n", optim.optstep, optim.object_f, optim.const_h[0], k);
    optim.design_s = xnew;
    running = !last;
  }
  return 0;
}
