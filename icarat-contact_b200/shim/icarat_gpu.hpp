// icarat_gpu.hpp -- ICARAT's analysis / filter / optimiser classes over the
// B200 library (libicarat_b200.so, C ABI in icarat_b200.h).
//
// A structured-box ICARAT app (opt-macro-oc, opt-mma-HelmholtzFilter) keeps its
// shape: the same class names, constructor arguments, call order and result
// fields, with Eigen and toml11 replaced by the small Eigen-free types below
// and the TOML subset reader of icarat_toml.hpp.
//
//   ICARAT                                        here
//   MeshIcarat<E,N>   (src/io/mesh_icarat.hpp:18-60)   same; generate() also
//                                                      creates the device problem
//   LinearElastic     (src/problem/elasticity.hpp:24-80) design / material
//                                                      accessors, volume, Ke()
//   BCIcarat<E,N>     (src/io/boundary_condition_icarat.hpp:30-60)
//                     input_dirich, makeDOF, input_neumann (+ `point` loads)
//   Force, Value      (src/problem/base.hpp:108-131)  VectorXd stand-in
//   LinearAnalysis<E,N>::solve(solvName, log)      (src/analysis/linear.hpp:15-104)
//   Filter<E,N>::densityFilter / threshold / thresholdDerivative
//                     (src/optimization/filter.hpp:17-185)
//   FilterHelmholtz<E,N>::densityFilter(x, solvName, log, sensFlag)
//                     (src/optimization/filter_helm.hpp:28-137)
//   OC::UpdateVariables (src/optimization/opt-solver/OCSolver.hpp:16-70)
//   MMASolver::Update (src/optimization/opt-solver/MMASolver.hpp:62-80)
//   GCMMASolver::OuterUpdate / InnerUpdate / ConCheck (GCMMASolver.hpp:60-90)
//   Optimize          (src/optimization/opt_base.hpp:14-76)
//
// Differences a caller sees:
//   * solver names: "Eigen_CG", "CG", "Scaling_CG" run the FP64 Jacobi-PCG with
//     Eigen's stopping rule (tol 1e-10, 10000 iterations, Solvers' defaults);
//     "Eigen_LDLT" (a direct solve in ICARAT) runs FP64 multigrid-PCG to 1e-12;
//     "GPU_FP64" / "GPU_MIXED" run FP64 / mixed-precision multigrid-PCG to the
//     tolerance of setTolerance() (1e-10 unless set).  Other names print
//     ICARAT's message and exit(1), as solvers.cpp:57-61 does.
//   * LinearAnalysis::K() does not exist (the operator is matrix-free); use
//     matvec() and diagonal().
//   * OC::UpdateVariables takes the volume callback of the apps
//     (opt_macro_oc.cpp:155-164: volume of threshold(filter(x+))) as an
//     OcVolume descriptor, because the bisection and the callback run on the
//     device together; an arbitrary host lambda is not accepted.
//   * sensitivities come from sensitivity() below (the device computes
//     -(E'/E) u_e^T Ke u_e and v_e), not from per-element Ke loops.
//   * device failures throw icarat::gpu_error (ICARAT has none to report).
//   * makeMisesStress computes every element's stress on the device once per
//     solve; solve() also fills node[].reaction.
#pragma once
#include <cmath>
#include <cstdlib>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "icarat_b200.h"
#include "icarat_toml.hpp"

namespace icarat
{
namespace toml = icarat_b200::toml;

class gpu_error : public std::runtime_error
{
public:
  gpu_error(int code, const std::string &what)
      : std::runtime_error(what + ": " + icb_last_error()), code_(code)
  {
  }
  int code() const { return code_; }

private:
  int code_;
};

inline void check(int rc, const char *what)
{
  if(rc != ICB_OK)
    throw gpu_error(rc, what);
}

/// the parts of Eigen::VectorXd the apps use on Force / Value
class VectorXd
{
public:
  explicit VectorXd(long n = 0) : v_(std::size_t(n), 0.0) {}
  long size() const { return long(v_.size()); }
  double *data() { return v_.data(); }
  const double *data() const { return v_.data(); }
  double &operator()(long i) { return v_[std::size_t(i)]; }
  double operator()(long i) const { return v_[std::size_t(i)]; }
  double &operator[](long i) { return v_[std::size_t(i)]; }
  double operator[](long i) const { return v_[std::size_t(i)]; }
  void setZero() { std::fill(v_.begin(), v_.end(), 0.0); }
  void resize(long n) { v_.assign(std::size_t(n), 0.0); }
  double dot(const VectorXd &o) const
  {
    double s = 0.0;
    for(std::size_t i = 0; i < v_.size(); i++)
      s += v_[i] * o.v_[i];
    return s;
  }
  double norm() const { return std::sqrt(dot(*this)); }

private:
  std::vector<double> v_;
};

namespace detail
{
/// the device objects behind one FEM problem
struct Device
{
  icb_ctx ctx = nullptr;
  icb_problem prob = nullptr;
  icb_grid_desc desc{};
  bool finalized = false;
  double volume = 0.0;        ///< element volume (uniform grid)
  std::vector<double> K0;     ///< unit-modulus element matrix
  long long solves = 0;       ///< solves so far
  long long stressOf = -1;    ///< the solve the cached stresses belong to
  std::vector<double> mises, stress;
  /// element stresses of the last solve, fetched once per solve
  void stresses(int voigt)
  {
    if(stressOf == solves)
      return;
    long long nel = 0;
    check(icb_problem_sizes(prob, &nel, nullptr, nullptr, nullptr), "icb_problem_sizes");
    mises.resize(std::size_t(nel));
    stress.resize(std::size_t(nel) * voigt);
    check(icb_von_mises(prob, mises.data(), stress.data()), "icb_von_mises");
    stressOf = solves;
  }
  Device() = default;
  Device(const Device &) = delete;
  Device &operator=(const Device &) = delete;
  ~Device()
  {
    if(prob)
      icb_problem_destroy(prob);
    if(ctx)
      icb_ctx_destroy(ctx);
  }
  void finalize()
  {
    if(finalized)
      return;
    long long numeq = 0;
    check(icb_finalize(prob, &numeq), "icb_finalize");
    finalized = true;
  }
};

inline int default_device()
{
  const char *e = std::getenv("ICB_DEVICE");
  return e ? std::atoi(e) : 0;
}

/// a context for objects ICARAT constructs without a FEM (MMASolver)
inline icb_ctx shared_context()
{
  static std::shared_ptr<std::remove_pointer<icb_ctx>::type> ctx = [] {
    icb_ctx c = nullptr;
    check(icb_ctx_create(default_device(), &c), "icb_ctx_create");
    return std::shared_ptr<std::remove_pointer<icb_ctx>::type>(c, icb_ctx_destroy);
  }();
  return ctx.get();
}

[[noreturn]] inline void fatal(const std::string &msg)
{
  std::cerr << msg << std::endl;
  std::exit(1);
}
} // namespace detail

/// problem sizes (src/problem/base.hpp:16-34) plus the device problem
struct FEM
{
  int neq = 0;   ///< total dof
  int numeq = 0; ///< number of equations (neq - Dirichlet DOFs)
  int ndim = 0;
  int nelx = 0;
  int voigt = 0;
  int dofnp = 0;
  int numnp = 0;
  int device = detail::default_device();  ///< CUDA device of the problem
  std::shared_ptr<detail::Device> gpu;    ///< set by MeshIcarat::generate
};

struct Dirichlet
{
  int flag[6] = {0, 0, 0, 0, 0, 0};
  double val[6] = {0, 0, 0, 0, 0, 0};
};
struct Neumann
{
  int flag[3] = {0, 0, 0};
  double val[3] = {0, 0, 0};
};

struct Element
{
  int numdof = 0;
  int ne = 0;
  int ipmax = 0;
  std::string eType;
  int ID = 0;
  std::vector<int> nodeID;
  double volume = 0.0;
};

struct Node
{
  int ID = 0;
  int dof[6] = {0, 0, 0, 0, 0, 0};
  double x[3] = {0, 0, 0};
  std::shared_ptr<Dirichlet> dirich;
  std::shared_ptr<Neumann> neum;
  double val[3] = {0, 0, 0};
  double reaction[3] = {0, 0, 0};
  double du[3] = {0, 0, 0};
};

struct Force
{
  explicit Force(int numeq) : fext_org(numeq), fext(numeq), fint(numeq), fres(numeq) {}
  VectorXd fext_org, fext, fint, fres;
};

struct Value
{
  explicit Value(int numeq) : val(numeq) {}
  VectorXd val;
};

/// SIMP linear-elastic element (elasticity.hpp:15-80, elasticity.cpp:19-32)
class LinearElastic : public Element
{
public:
  LinearElastic(int voigt, int ne_, int ipmax_, int numdof_) : voigt_(voigt)
  {
    ne = ne_;
    ipmax = ipmax_;
    numdof = numdof_;
  }
  void setParameter(const toml::value &config)
  {
    const toml::value &mat = toml::find(config, "material");
    if(toml::find<std::string>(mat, "type") != "Elastic")
      detail::fatal("Error: [material] type must be \"Elastic\"");
    design_s_ = toml::find<double>(mat, "designs_0");
    pp_ = toml::find<double>(mat, "penalty");
    auto y = toml::find<std::array<double, 2>>(mat, "young");
    young1_ = y[0];
    young2_ = y[1];
    poisson_ = toml::find<double>(mat, "poisson");
    mattype_ = toml::find<std::string>(mat, "state");
    if(toml::find<int>(config, "mesh", "dimension") == 3)
      mattype_ = "3D";
  }
  double design_s() const { return design_s_; }
  void setDesignS(double &d) { design_s_ = d; }
  double young1() const { return young1_; }
  double young2() const { return young2_; }
  double pp() const { return pp_; }
  double poisson() const { return poisson_; }
  const std::string &mattype() const { return mattype_; }
  /// SIMP (elasticity.hpp:15-22)
  double young() const
  {
    double rp = std::pow(design_s_, pp_);
    return (1.0 - rp) * young1_ + rp * young2_;
  }
  /// Ke = E(rho) K0, row-major numdof x numdof (makeKeFint on a uniform grid);
  /// K0 is the problem's (set by MeshIcarat::generate)
  std::vector<double> Ke() const
  {
    std::vector<double> k(K0_ ? *K0_ : std::vector<double>());
    double E = young();
    for(double &v : k)
      v *= E;
    return k;
  }
  void attachK0(std::shared_ptr<const std::vector<double>> k0) { K0_ = std::move(k0); }

  /// Elastic::makeMisesStress (elasticity.cpp:165-208): the element's stress
  /// and von Mises value from the last solve (all elements are computed on
  /// the device on the first call after a solve)
  template <class N> void makeMisesStress(FEM &fem, std::vector<N> &)
  {
    fem.gpu->stresses(voigt_);
    mises_ = fem.gpu->mises[std::size_t(ID)];
    stress_.assign(fem.gpu->stress.begin() + std::size_t(ID) * voigt_,
                   fem.gpu->stress.begin() + std::size_t(ID + 1) * voigt_);
  }
  double mises() const { return mises_; }
  const std::vector<double> &stress() const { return stress_; }

private:
  int voigt_;
  double mises_ = 0.0;
  std::vector<double> stress_;
  double design_s_ = 0.0, pp_ = 3.0, young1_ = 0.0, young2_ = 1.0, poisson_ = 0.3;
  std::string mattype_ = "plane_stress";
  std::shared_ptr<const std::vector<double>> K0_;
};

namespace detail
{
inline int state_of(const std::string &s)
{
  if(s == "plane_stress")
    return ICB_PLANE_STRESS;
  if(s == "plane_strain")
    return ICB_PLANE_STRAIN;
  if(s == "3D")
    return ICB_3D;
  fatal("Error: unknown material state \"" + s + "\"");
}
} // namespace detail

/// structured box mesh (src/io/mesh_icarat.hpp:18-128, 320-614; quad4 and hexa8)
template <class E, class N> class MeshIcarat
{
public:
  MeshIcarat(FEM &fem, const toml::value &config) : fem_(fem), config_(config) {}

  void setParameter(std::string probType)
  {
    if(probType != "structure")
      detail::fatal("Error: MeshIcarat supports the \"structure\" problem type only");
    const toml::value &mesh = toml::find(config_, "mesh");
    fem_.ndim = toml::find<int>(mesh, "dimension");
    fem_.dofnp = fem_.ndim;
    fem_.voigt = fem_.ndim == 2 ? 3 : 6;
    type_ = toml::find<std::string>(mesh, "type");
    if(!((type_ == "quad4" && fem_.ndim == 2) || (type_ == "hexa8" && fem_.ndim == 3)))
      detail::fatal("Error: mesh type \"" + type_ + "\" is not available (quad4 in 2D, hexa8 in 3D)");
    ne_ = fem_.ndim == 2 ? 4 : 8;
    ipmax_ = ne_;
    div_ = toml::find<std::array<int, 3>>(mesh, "division");
    length_ = toml::find<std::array<double, 3>>(mesh, "length");
    long long nx = div_[0], ny = div_[1], nz = fem_.ndim == 3 ? div_[2] : 0;
    fem_.numnp = int((nx + 1) * (ny + 1) * (nz + 1));
    fem_.neq = fem_.numnp * fem_.dofnp;
    fem_.nelx = int(nx * ny * (fem_.ndim == 3 ? nz : 1));
    nelx_ = fem_.nelx;
  }

  int numeleTypes() { return 1; }
  const int &nelx(int) const { return nelx_; }
  const int &ne(int) const { return ne_; }
  const int &ipmax(int) const { return ipmax_; }
  const std::array<int, 3> &div() const { return div_; }
  const std::array<double, 3> &length() const { return length_; }

  /// element IDs and connectivity, node IDs and coordinates (meshBox), and
  /// the device problem with the material of element[0]
  void generate(std::vector<E> &element, std::vector<N> &node)
  {
    if((int)element.size() != fem_.nelx || (int)node.size() != fem_.numnp)
      detail::fatal("Error: element / node vectors do not match the mesh");
    const int d = fem_.ndim;
    const long long nx = div_[0], ny = div_[1], nz = d == 3 ? div_[2] : 1;
    const long long sx = nx + 1, sxy = sx * (ny + 1);
    for(long long n = 0; n < fem_.numnp; n++)
    {
      N &q = node[n];
      q.ID = int(n);
      long long i = n % sx, j = (n / sx) % (ny + 1), k = n / sxy;
      q.x[0] = length_[0] / double(nx) * double(i);
      q.x[1] = length_[1] / double(ny) * double(j);
      q.x[2] = d == 3 ? length_[2] / double(nz) * double(k) : 0.0;
    }
    for(long long e = 0; e < fem_.nelx; e++)
    {
      E &el = element[e];
      el.ID = int(e);
      el.eType = type_;
      long long i = e % nx, j = (e / nx) % ny, k = e / (nx * ny);
      long long b = i + j * sx + (d == 3 ? k * sxy : 0);
      long long nd[4] = {b, b + 1, b + 1 + sx, b + sx};
      el.nodeID.clear();
      for(long long v : nd)
        el.nodeID.push_back(int(v));
      if(d == 3)
        for(long long v : nd)
          el.nodeID.push_back(int(v + sxy));
    }
    auto dev = std::make_shared<detail::Device>();
    const E &e0 = element.at(0);
    icb_grid_desc &g = dev->desc;
    g.dim = d;
    g.nx = int(nx);
    g.ny = int(ny);
    g.nz = d == 3 ? int(nz) : 1;
    g.lx = length_[0];
    g.ly = length_[1];
    g.lz = d == 3 ? length_[2] : 1.0;
    g.state = detail::state_of(e0.mattype());
    g.young1 = e0.young1();
    g.young2 = e0.young2();
    g.poisson = e0.poisson();
    g.penalty = e0.pp();
    check(icb_ctx_create(fem_.device, &dev->ctx), "icb_ctx_create");
    check(icb_problem_create(dev->ctx, &g, &dev->prob), "icb_problem_create");
    check(icb_element_volume(dev->prob, &dev->volume), "icb_element_volume");
    int nd = ne_ * d;
    dev->K0.assign(std::size_t(nd) * nd, 0.0);
    check(icb_get_K0(dev->prob, dev->K0.data()), "icb_get_K0");
    auto k0 = std::make_shared<const std::vector<double>>(dev->K0);
    for(long long e = 0; e < fem_.nelx; e++)
    {
      element[e].volume = dev->volume;
      element[e].attachK0(k0);
    }
    fem_.gpu = dev;
  }

private:
  FEM &fem_;
  const toml::value &config_;
  std::string type_;
  int nelx_ = 0, ne_ = 0, ipmax_ = 0;
  std::array<int, 3> div_{};
  std::array<double, 3> length_{};
};

/// boundary conditions from TOML (src/io/boundary_condition_icarat.hpp:30-396)
template <class E, class N> class BCIcarat
{
public:
  BCIcarat(FEM &fem, std::vector<E> &element, std::vector<N> &node)
      : fem(fem), element(element), node(node)
  {
    if(!fem.gpu)
      detail::fatal("Error: call MeshIcarat::generate before BCIcarat");
  }

  /// dirichlet = [[flag x6], [val x6], [[xmin,xmax],[ymin,ymax],[zmin,zmax]]], ...
  void input_dirich(const toml::value &config)
  {
    const toml::array &rows = toml::find<toml::array>(config, "boundary_condition", "dirichlet");
    for(const toml::value &r : rows)
    {
      const toml::array &t = r.as_array();
      if(t.size() != 3)
        detail::fatal("Error: a dirichlet row needs [flags], [values], [range]");
      auto flag = toml::get<std::array<int, 6>>(t[0]);
      auto val = toml::get<std::array<double, 6>>(t[1]);
      auto rng = toml::get<std::array<std::array<double, 2>, 3>>(t[2]);
      double range[6] = {rng[0][0], rng[0][1], rng[1][0], rng[1][1], rng[2][0], rng[2][1]};
      check(icb_dirichlet_box(fem.gpu->prob, flag.data(), val.data(), range), "icb_dirichlet_box");
    }
  }

  /// countDOF numbering into node[].dof; returns numeq
  int makeDOF()
  {
    long long numeq = 0;
    std::vector<int> dof(fem.neq);
    check(icb_count_dof(fem.gpu->prob, dof.data(), &numeq), "icb_count_dof");
    for(int n = 0; n < fem.numnp; n++)
    {
      bool any = false;
      for(int c = 0; c < fem.dofnp; c++)
      {
        node[n].dof[c] = dof[std::size_t(n) * fem.dofnp + c];
        any = any || node[n].dof[c] >= numeq;
      }
      if(any)
      {
        node[n].dirich = std::make_shared<Dirichlet>();
        for(int c = 0; c < fem.dofnp; c++)
          node[n].dirich->flag[c] = node[n].dof[c] >= numeq ? 1 : 0;
      }
    }
    return int(numeq);
  }

  /// neumann = [[val x3], [[xmin,xmax],[ymin,ymax],[zmin,zmax]]], ... (constant
  /// tractions on element sides); the extension key `point` =
  /// [[fx,fy,fz], [x,y,z]], ... adds nodal point loads at the nodes within
  /// 1e-7 of (x,y,z).  Fills force.fext_org and freezes the problem.
  void input_neumann(const toml::value &config, Force &force)
  {
    const toml::value &bc = toml::find(config, "boundary_condition");
    if(bc.contains("neumann"))
      for(const toml::value &r : bc.at("neumann").as_array())
      {
        const toml::array &t = r.as_array();
        if(t.size() != 2)
          detail::fatal("Error: a neumann row needs [values], [range]");
        auto val = toml::get<std::array<double, 3>>(t[0]);
        auto rng = toml::get<std::array<std::array<double, 2>, 3>>(t[1]);
        double range[6] = {rng[0][0], rng[0][1], rng[1][0], rng[1][1], rng[2][0], rng[2][1]};
        check(icb_traction_box(fem.gpu->prob, val.data(), range), "icb_traction_box");
      }
    if(bc.contains("point"))
      for(const toml::value &r : bc.at("point").as_array())
      {
        const toml::array &t = r.as_array();
        auto f = toml::get<std::array<double, 3>>(t.at(0));
        auto x = toml::get<std::array<double, 3>>(t.at(1));
        for(const N &q : node)
          if(std::fabs(q.x[0] - x[0]) <= 1e-7 && std::fabs(q.x[1] - x[1]) <= 1e-7 &&
             std::fabs(q.x[2] - x[2]) <= 1e-7)
            check(icb_nodal_load(fem.gpu->prob, q.ID, f.data()), "icb_nodal_load");
      }
    fem.gpu->finalize();
    if(force.fext_org.size() != fem.numeq)
      detail::fatal("Error: Force was not built with makeDOF()'s numeq");
    check(icb_get_load(fem.gpu->prob, force.fext_org.data()), "icb_get_load");
    force.fext = force.fext_org;
  }

private:
  FEM &fem;
  std::vector<E> &element;
  std::vector<N> &node;
};

/// LinearAnalysis<E,N> (src/analysis/linear.hpp:15-166), matrix-free on the device
template <class E, class N> class LinearAnalysis
{
public:
  LinearAnalysis(FEM &fem, std::vector<E> &element, std::vector<N> &node, Force &force,
                 Value &value)
      : fem(fem), element(element), node(node), force(force), value(value)
  {
    if(!fem.gpu)
      detail::fatal("Error: call MeshIcarat::generate before LinearAnalysis");
  }

  /// tolerance and iteration cap of the "GPU_*" solver names
  void setTolerance(double tol, int maxit)
  {
    tol_ = tol;
    maxit_ = maxit;
  }

  void solve(std::string solvName, bool log)
  {
    icb_solve_opts o{};
    o.precision = ICB_FP64;
    o.precond = ICB_PRECOND_JACOBI;
    o.tol = 1e-10;
    o.maxit = 10000;
    if(solvName == "Eigen_CG" || solvName == "CG" || solvName == "Scaling_CG")
    {
    }
    else if(solvName == "Eigen_LDLT")
    {
      o.precond = ICB_PRECOND_GMG;
      o.tol = 1e-12;
      o.maxit = 20000;
    }
    else if(solvName == "GPU_FP64" || solvName == "GPU_MIXED" || solvName == "GPU_JACOBI")
    {
      o.precision = solvName == "GPU_MIXED" ? ICB_MIXED : ICB_FP64;
      o.precond = solvName == "GPU_JACOBI" ? ICB_PRECOND_JACOBI : ICB_PRECOND_GMG;
      o.tol = tol_;
      o.maxit = maxit_;
    }
    else
      detail::fatal("Error ! Solver type name is wrong.");
    detail::Device &g = *fem.gpu;
    g.finalize();
    rho_.resize(element.size());
    for(std::size_t e = 0; e < element.size(); e++)
      rho_[e] = element[e].design_s();
    check(icb_set_density(g.prob, rho_.data()), "icb_set_density");
    int rc = icb_solve(g.prob, &o, &info_);
    if(rc == ICB_ERR_MAXITER)
    {
      if(log)
        std::cout << "not converge: " << info_.iters << " iterations, relres " << info_.relres
                  << std::endl;
    }
    else
      check(rc, "icb_solve");
    force.fext = force.fext_org;
    g.solves++;
    check(icb_get_displacement(g.prob, value.val.data()), "icb_get_displacement");
    nodeval_.resize(std::size_t(fem.neq));
    check(icb_get_node_values(g.prob, nodeval_.data()), "icb_get_node_values");
    for(int n = 0; n < fem.numnp; n++)
      for(int c = 0; c < 3; c++)
        node[n].val[c] = c < fem.dofnp ? nodeval_[std::size_t(n) * fem.dofnp + c] : 0.0;
    // node[].reaction (linear.hpp:89-91)
    check(icb_reactions(g.prob, nodeval_.data()), "icb_reactions");
    for(int n = 0; n < fem.numnp; n++)
      for(int c = 0; c < 3; c++)
        node[n].reaction[c] = c < fem.dofnp ? nodeval_[std::size_t(n) * fem.dofnp + c] : 0.0;
    if(log)
      std::cout << "#iterations: " << info_.iters << "  estimated error: " << info_.relres
                << "  true ||f-Ku||/||f||: " << info_.true_relres << std::endl;
  }

  /// y = K x over free DOFs (numeq), the product ICARAT forms with K()
  void matvec(const VectorXd &x, VectorXd &y) const
  {
    check(icb_matvec(fem.gpu->prob, x.data(), y.data()), "icb_matvec");
  }
  void diagonal(VectorXd &d) const { check(icb_diagonal(fem.gpu->prob, d.data()), "icb_diagonal"); }
  const icb_solve_info &info() const { return info_; }

private:
  FEM &fem;
  std::vector<E> &element;
  std::vector<N> &node;
  Force &force;
  Value &value;
  double tol_ = 1e-10;
  int maxit_ = 20000;
  icb_solve_info info_{};
  std::vector<double> rho_, nodeval_;
};

/// dc_e = -(E'/E) u_e^T Ke u_e and dv_e = v_e (the apps' sensitivity(),
/// opt_macro_oc.cpp:182-212) from the last solve; dv may be NULL
inline void sensitivity(const FEM &fem, std::vector<double> &dc, std::vector<double> *dv)
{
  dc.resize(std::size_t(fem.nelx));
  if(dv)
    dv->resize(std::size_t(fem.nelx));
  check(icb_sensitivity(fem.gpu->prob, dc.data(), dv ? dv->data() : nullptr), "icb_sensitivity");
}

namespace detail
{
inline std::vector<double> threshold(const std::vector<double> &x, double beta, double T,
                                      bool deriv)
{
  std::vector<double> out(x.size());
  check(icb_threshold(shared_context(), (long long)x.size(), x.data(), beta, T,
                      deriv ? nullptr : out.data(), deriv ? out.data() : nullptr),
        "icb_threshold");
  return out;
}
} // namespace detail

/// cone density filter (src/optimization/filter.hpp:17-185)
template <class E, class N> class Filter
{
public:
  Filter(FEM &fem_, std::vector<E> &, std::vector<N> &, double radius_) : fem(fem_)
  {
    check(icb_cone_create(fem.gpu->prob, radius_, &h_), "icb_cone_create");
  }
  ~Filter() { icb_cone_destroy(h_); }
  Filter(const Filter &) = delete;
  Filter &operator=(const Filter &) = delete;

  std::vector<double> densityFilter(const std::vector<double> &x, bool isSens)
  {
    std::vector<double> out(x.size());
    check(icb_cone_filter(h_, x.data(), out.data(), isSens ? 1 : 0), "icb_cone_filter");
    return out;
  }
  std::vector<double> threshold(const std::vector<double> &x, double beta, double T)
  {
    return detail::threshold(x, beta, T, false);
  }
  std::vector<double> thresholdDerivative(const std::vector<double> &x, double beta, double T)
  {
    return detail::threshold(x, beta, T, true);
  }
  icb_cone handle() const { return h_; }

private:
  FEM &fem;
  icb_cone h_ = nullptr;
};

/// PDE (Helmholtz) density filter (src/optimization/filter_helm.hpp:28-256)
template <class E, class N> class FilterHelmholtz
{
public:
  FilterHelmholtz(FEM &fem_, std::vector<E> &, std::vector<N> &, double radious_) : fem(fem_)
  {
    check(icb_helm_create(fem.gpu->prob, radious_, &h_), "icb_helm_create");
  }
  ~FilterHelmholtz() { icb_helm_destroy(h_); }
  FilterHelmholtz(const FilterHelmholtz &) = delete;
  FilterHelmholtz &operator=(const FilterHelmholtz &) = delete;

  /// solvName / log are accepted for the call shape; the device solve is
  /// Jacobi-PCG to 1e-10 (the Eigen_CG default the apps use)
  std::vector<double> densityFilter(const std::vector<double> &x, std::string, int,
                                    bool sensFlag)
  {
    std::vector<double> out(x.size());
    check(icb_helm_filter(h_, x.data(), out.data(), sensFlag ? 1 : 0), "icb_helm_filter");
    return out;
  }
  std::vector<double> threshold(const std::vector<double> &x, double beta, double T)
  {
    return detail::threshold(x, beta, T, false);
  }
  std::vector<double> thresholdDerivative(const std::vector<double> &x, double beta, double T)
  {
    return detail::threshold(x, beta, T, true);
  }

private:
  FEM &fem;
  icb_helm h_ = nullptr;
};

/// the volume callback of opt_macro_oc.cpp:155-164 as data: the device OC
/// evaluates sum_e threshold(filter(x+))_e v_e inside its bisection
struct OcVolume
{
  icb_problem prob;
  icb_cone cone; ///< NULL: no filter
  double beta;   ///< <= 0: no threshold
  double T;
};
template <class E, class N> OcVolume oc_volume(const FEM &fem, const Filter<E, N> &f, double beta,
                                               double T)
{
  return OcVolume{fem.gpu->prob, f.handle(), beta, T};
}

/// OC (src/optimization/opt-solver/OCSolver.hpp:16-80)
class OC
{
public:
  explicit OC(int n) : n_(n) {}
  void setMoveLimit(double m) { move_ = m; }

  void UpdateVariables(std::vector<double> &xk, std::vector<double> &dfdx, double g,
                       std::vector<double> &dgdx, std::vector<double> &xmin,
                       std::vector<double> &xmax, const OcVolume &gkp1)
  {
    if((int)xk.size() != n_)
      detail::fatal("Error: OC size mismatch");
    int steps = 0;
    check(icb_oc_update(gkp1.prob, gkp1.cone, xk.data(), dfdx.data(), g, dgdx.data(), xmin.data(),
                        xmax.data(), move_, gkp1.beta, gkp1.T, &steps),
          "icb_oc_update");
    steps_ = steps;
  }
  int lastBisections() const { return steps_; }

private:
  int n_;
  double move_ = 0.15;
  int steps_ = 0;
};

/// MMASolver (src/optimization/opt-solver/MMASolver.hpp:62-117), one constraint
class MMASolver
{
public:
  MMASolver(int n, int m, double a = 0.0, double c = 100000.0, double d = 0.0)
  {
    if(m != 1 || a != 0.0 || c != 100000.0 || d != 0.0)
      detail::fatal("Error: the device MMA solves m = 1 with a = 0, c = 1e5, d = 0");
    check(icb_mma_create(detail::shared_context(), n, m, &h_), "icb_mma_create");
  }
  ~MMASolver() { icb_mma_destroy(h_); }
  MMASolver(const MMASolver &) = delete;
  MMASolver &operator=(const MMASolver &) = delete;

  void Update(double *xval, const double *dfdx, const double *gx, const double *dgdx,
              const double *xmin, const double *xmax)
  {
    check(icb_mma_update(h_, xval, dfdx, gx, dgdx, xmin, xmax), "icb_mma_update");
  }

private:
  icb_mma h_ = nullptr;
};

/// GCMMASolver (src/optimization/opt-solver/GCMMASolver.hpp:60-90), one
/// constraint: OuterUpdate, InnerUpdate, ConCheck on the device
class GCMMASolver
{
public:
  GCMMASolver(int n, int m, double a = 0.0, double c = 1000.0, double d = 0.0)
  {
    if(m != 1 || a != 0.0 || c != 1000.0 || d != 0.0)
      detail::fatal("Error: the device GCMMA solves m = 1 with a = 0, c = 1000, d = 0");
    check(icb_gcmma_create(detail::shared_context(), n, m, &h_), "icb_gcmma_create");
  }
  ~GCMMASolver() { icb_gcmma_destroy(h_); }
  GCMMASolver(const GCMMASolver &) = delete;
  GCMMASolver &operator=(const GCMMASolver &) = delete;

  void OuterUpdate(double *xmma, const double *xval, double f0x, const double *df0dx,
                   const double *fx, const double *dfdx, const double *xmin, const double *xmax)
  {
    check(icb_gcmma_outer(h_, xmma, xval, f0x, df0dx, fx, dfdx, xmin, xmax), "icb_gcmma_outer");
  }
  void InnerUpdate(double *xmma, double f0xnew, const double *fxnew, const double *xval,
                   double f0x, const double *df0dx, const double *fx, const double *dfdx,
                   const double *xmin, const double *xmax)
  {
    check(icb_gcmma_inner(h_, xmma, f0xnew, fxnew, xval, f0x, df0dx, fx, dfdx, xmin, xmax),
          "icb_gcmma_inner");
  }
  bool ConCheck(double f0xnew, const double *fxnew) const
  {
    int ok = 0;
    check(icb_gcmma_concheck(h_, f0xnew, fxnew, &ok), "icb_gcmma_concheck");
    return ok != 0;
  }

private:
  icb_gcmma h_ = nullptr;
};

/// design-variable bookkeeping (src/optimization/opt_base.hpp:14-76)
class Optimize
{
public:
  Optimize(int design, int constraint, double xmin_, double xmax_)
      : design_s(design), const_h(constraint), dfds(design), dgds(constraint * design),
        xmin(design, xmin_), xmax(design, xmax_)
  {
  }
  /// 0 once |f_old - f| / f < epsilon after minstep steps, else 1
  int isConvergence(double epsilon, double minstep)
  {
    if(std::fabs(object_old - object_f) / object_f < epsilon && optstep > minstep)
      return 0;
    object_old = object_f;
    return 1;
  }
  std::vector<double> design_s, const_h, dfds, dgds, xmin, xmax;
  double object_f = 0.0, object_old = 0.0;
  int optstep = 0;
};

} // namespace icarat
