// opt_macro_mma_nondesign_gpu.cpp -- ICARAT's opt-macro-mma-nondesign app
// (opt-macro-mma-nondesign/opt_macro_mma_nondesign.cpp:14-178, 222-309) on the
// B200 shim: cone filter, threshold, linear analysis, stresses, volume
// constraint over the design elements, sensitivities, adjoint filter,
// non-design sensitivities set to 0, MMA update.  One line per step on stdout:
// "step,compliance,constraint,max von Mises"; with [this_problem] output =
// true also res<step>.vtk (displacement, density, mises) and function.csv.
//
// usage: opt_macro_mma_nondesign_gpu <config.toml>
// [this_problem]: filterR (required), non_design = [[[value], [[x0,x1],
// [y0,y1],[z0,z1]]], ...] (required), steps (fixed count; default the app's
// isConvergence(1e-5, 50) rule, at most 1000 steps), solver ("Eigen_CG"),
// output (false).
//
// Element selection follows the app: an element whose centre lies strictly
// inside a row's box takes the row's value as its initial design and joins
// the non-design list; an element outside ANY row's box joins the design
// list (so with several rows an element can be in both lists, as in the
// app).  In 3D the app compares centreZ with range[2][2], one past the end of
// the [z0, z1] pair; here the upper z bound is z1.
#include <algorithm>
#include <cstdio>
#include <fstream>

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

void designIds(FEM &fem, std::vector<LinearElastic> &element, std::vector<Node> &node,
               const toml::value &config, std::vector<int> &design, std::vector<int> &nondesign)
{
  for(const toml::value &row : toml::find<toml::array>(config, "this_problem", "non_design"))
  {
    const toml::array &t = row.as_array();
    double value = toml::get<std::array<double, 1>>(t.at(0))[0];
    auto r = toml::get<std::array<std::array<double, 2>, 3>>(t.at(1));
    for(int i = 0; i < fem.nelx; i++)
    {
      double c[3] = {0, 0, 0};
      for(int j = 0; j < element[i].ne; j++)
        for(int k = 0; k < 3; k++)
          c[k] += node[element[i].nodeID[j]].x[k] / element[i].ne;
      bool in = r[0][0] < c[0] && c[0] < r[0][1] && r[1][0] < c[1] && c[1] < r[1][1];
      if(fem.ndim == 3)
        in = in && r[2][0] < c[2] && c[2] < r[2][1];
      if(in)
      {
        nondesign.push_back(i);
        element[i].setDesignS(value);
      }
      else
        design.push_back(i);
    }
  }
  for(auto *v : {&design, &nondesign})
  {
    std::sort(v->begin(), v->end());
    v->erase(std::unique(v->begin(), v->end()), v->end());
  }
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
  const std::string solver = option<std::string>(config, "solver", "Eigen_CG");
  const bool output = option<bool>(config, "output", false);
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

  std::vector<int> designIDs, nondesignIDs;
  designIds(fem, element, node, config, designIDs, nondesignIDs);

  Optimize optim(fem.nelx, 1, 1.0e-4, 1.0);
  MMASolver mma(fem.nelx, 1);
  Filter<LinearElastic, Node> filter(fem, element, node, filterR);
  for(int i = 0; i < fem.nelx; i++)
    optim.design_s[i] = element[i].design_s();
  LinearAnalysis<LinearElastic, Node> compt(fem, element, node, force, dis);

  double V0 = 0.0;
  std::vector<double> dv;
  for(int running = 1; running;)
  {
    optim.optstep++;
    std::vector<double> xf = filter.densityFilter(optim.design_s, false);
    const double beta = std::min(std::pow(2.0, optim.optstep / 40), 16.0);
    std::vector<double> xh = filter.threshold(xf, beta, T);
    std::vector<double> dxh = filter.thresholdDerivative(xf, beta, T);
    for(int i = 0; i < fem.nelx; i++)
      element[i].setDesignS(xh[i]);

    compt.solve(solver, false);
    double smax = 0.0;
    for(auto &e : element)
    {
      e.makeMisesStress(fem, node);
      smax = std::max(smax, e.mises());
    }
    optim.object_f = dis.val.dot(force.fext);

    double vs = 0.0;
    for(int i : designIDs)
      vs += element[i].design_s() * element[i].volume;
    if(optim.optstep == 1)
    {
      V0 = vs;
      optim.const_h[0] = 0.0;
    }
    else
      optim.const_h[0] = vs / V0 - 1.0;
    std::printf("%d,%.17g,%.17g,%.17g\n", optim.optstep, optim.object_f, optim.const_h[0], smax);

    if(output)
    {
      addPlot(optim.optstep, optim.object_f, "function.csv", optim.optstep);
      std::ofstream fout("res" + std::to_string(optim.optstep) + ".vtk");
      makeHeaderVTK(fout);
      setPointVTK(node, fout);
      setElementVTK(element, fout);
      setElementTypeVTK(fem.ndim, element, fout);
      addPointVectorVTK("displacement", node, fout, true, [](Node &n) { return n.val; });
      addElementScalarVTK("density", element, fout, true,
                          [](LinearElastic &e) { return e.design_s(); });
      addElementScalarVTK("mises", element, fout, false, [](LinearElastic &e) { return e.mises(); });
    }

    running = fixedSteps > 0 ? optim.optstep < fixedSteps
                             : (optim.isConvergence(1.0e-5, 50) && optim.optstep < 1000);
    if(!running)
      break;

    sensitivity(fem, optim.dfds, &dv);
    for(int i = 0; i < fem.nelx; i++)
    {
      optim.dfds[i] *= dxh[i];
      optim.dgds[i] = dv[i] / V0 * dxh[i];
    }
    optim.dfds = filter.densityFilter(optim.dfds, true);
    optim.dgds = filter.densityFilter(optim.dgds, true);
    for(int i : nondesignIDs)
    {
      optim.dfds[i] = 0.0;
      optim.dgds[i] = 0.0;
    }
    mma.Update(optim.design_s.data(), optim.dfds.data(), optim.const_h.data(), optim.dgds.data(),
               optim.xmin.data(), optim.xmax.data());
  }
  return 0;
}
