"""The shim's result writers (legacy VTK, function.csv) produce ICARAT's
text layout: checked on a 2 x 1 quad mesh without a GPU."""
import os
import subprocess

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = r'''
#include <array>
#include <fstream>
#include <vector>
#include "icarat_export.hpp"
struct N { int ID; double x[3]; double val[3]; };
struct E { int ne; std::vector<int> nodeID; double d; };
int main()
{
  std::vector<N> node(6);
  for(int n = 0; n < 6; n++)
    node[n] = N{n, {double(n % 3), double(n / 3), 0.0}, {0.5 * n, -0.25 * n, 0.0}};
  std::vector<E> el = {E{4, {0, 1, 4, 3}, 0.25}, E{4, {1, 2, 5, 4}, 1.0}};
  std::ofstream f("res1.vtk");
  icarat::makeHeaderVTK(f);
  icarat::setPointVTK(node, f);
  icarat::setElementVTK(el, f);
  icarat::setElementTypeVTK(2, el, f);
  icarat::addPointVectorVTK("displacement", node, f, true, [](N &n) { return n.val; });
  icarat::addElementScalarVTK("density", el, f, true, [](E &e) { return e.d; });
  icarat::addElementScalarVTK("mises", el, f, false, [](E &e) { return 2.0 * e.d; });
  f.close();
  icarat::addPlot(1, 10.5, "function.csv", 1);
  icarat::addPlot(2, 9.25, "function.csv", 2);
  return 0;
}
'''

EXPECTED = (
    "# vtk DataFile Version 4.1\nvtk output\nASCII\nDATASET UNSTRUCTURED_GRID\n"
    "\nPOINTS\t6\tfloat\n"
    "0\t0\t0\t\n1\t0\t0\t\n2\t0\t0\t\n0\t1\t0\t\n1\t1\t0\t\n2\t1\t0\t\n"
    "\nCELLS 2\t10\n4\t0\t1\t4\t3\t\n4\t1\t2\t5\t4\t\n"
    "\nCELL_TYPES\t2\n9\n9\n"
    "\nPOINT_DATA\t6\nVECTORS displacement float\n"
    "0\t-0\t0\t\n0.5\t-0.25\t0\t\n1\t-0.5\t0\t\n1.5\t-0.75\t0\t\n2\t-1\t0\t\n2.5\t-1.25\t0\t\n"
    "\nCELL_DATA\t2\nSCALARS density float\nLOOKUP_TABLE default\n0.25\n1\n"
    "SCALARS mises float\nLOOKUP_TABLE default\n0.5\n2\n")


def test_vtk_and_graph_layout(tmp_path):
    src = tmp_path / "w.cpp"
    src.write_text(SRC)
    exe = tmp_path / "w"
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror",
                    "-I" + os.path.join(REPO, "icarat-contact_b200", "shim"), str(src), "-o",
                    str(exe)], check=True)
    subprocess.run([str(exe)], cwd=tmp_path, check=True)
    assert (tmp_path / "res1.vtk").read_text() == EXPECTED
    assert (tmp_path / "function.csv").read_text() == "1 10.5\n2 9.25\n"
