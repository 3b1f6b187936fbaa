// icarat_export.hpp -- result files of ICARAT's apps: legacy-VTK
// unstructured grids (src/io/export_vtk.hpp) and the plain-text graphs
// (src/io/export_graph.hpp), same call shapes and the same text layout
// (tab-separated fields, POINT_DATA / CELL_DATA headers on the first array),
// so res<step>.vtk and function.csv from the B200 apps open in the same tools.
// Lines end with '\n' (no per-line flush); values are written with the
// stream's default precision, as ICARAT's writers do.
#pragma once
#include <cassert>
#include <fstream>
#include <string>
#include <vector>

namespace icarat
{
/// VTK cell type of an element with ne nodes (export_vtk.hpp:15-42)
inline int cellTypes(int ndim, int ne)
{
  if(ndim == 2)
    switch(ne)
    {
    case 3: return 5;
    case 6: return 22;
    case 4: return 9;
    case 8: return 23;
    }
  else
    switch(ne)
    {
    case 4: return 10;
    case 8: return 12;
    case 6: return 13;
    case 20: return 25;
    case 15: return 26;
    }
  return 0;
}

inline void makeHeaderVTK(std::ofstream &out)
{
  out << "# vtk DataFile Version 4.1\nvtk output\nASCII\nDATASET UNSTRUCTURED_GRID\n";
}

template <class N> void setPointVTK(std::vector<N> &nodes, std::ofstream &out)
{
  out << "\nPOINTS\t" << nodes.size() << "\tfloat\n";
  for(const N &n : nodes)
    out << n.x[0] << "\t" << n.x[1] << "\t" << n.x[2] << "\t\n";
}

template <class E> void setElementVTK(std::vector<E> &elements, std::ofstream &out)
{
  std::size_t count = 0;
  for(const E &e : elements)
    count += e.nodeID.size() + 1;
  out << "\nCELLS " << elements.size() << "\t" << count << "\n";
  for(const E &e : elements)
  {
    out << e.nodeID.size() << "\t";
    for(int id : e.nodeID)
      out << id << "\t";
    out << "\n";
  }
}

template <class E> void setElementTypeVTK(int ndim, std::vector<E> &elements, std::ofstream &out)
{
  out << "\nCELL_TYPES\t" << elements.size() << "\n";
  for(const E &e : elements)
    out << cellTypes(ndim, e.ne) << "\n";
}

template <class N, class F>
void addPointScalarVTK(std::string name, std::vector<N> &nodes, std::ofstream &out, bool header,
                       F value)
{
  if(header)
    out << "\nPOINT_DATA\t" << nodes.size() << "\n";
  out << "SCALARS " << name << " float\nLOOKUP_TABLE default\n";
  for(N &n : nodes)
    out << value(n) << "\n";
}

template <class N, class F>
void addPointVectorVTK(std::string name, std::vector<N> &nodes, std::ofstream &out, bool header,
                       F values)
{
  if(header)
    out << "\nPOINT_DATA\t" << nodes.size() << "\n";
  out << "VECTORS " << name << " float\n";
  for(N &n : nodes)
  {
    const auto &v = values(n);
    out << v[0] << "\t" << v[1] << "\t" << v[2] << "\t\n";
  }
}

template <class E, class F>
void addElementScalarVTK(std::string name, std::vector<E> &elements, std::ofstream &out,
                         bool header, F value)
{
  if(header)
    out << "\nCELL_DATA\t" << elements.size() << "\n";
  out << "SCALARS " << name << " float\nLOOKUP_TABLE default\n";
  for(E &e : elements)
    out << value(e) << "\n";
}

template <class E, class F>
void addElementVectorVTK(std::string name, std::vector<E> &elements, std::ofstream &out,
                         bool header, F values)
{
  if(header)
    out << "\nCELL_DATA\t" << elements.size() << "\n";
  out << "VECTORS " << name << " float\n";
  for(E &e : elements)
  {
    const auto &v = values(e);
    out << v[0] << "\t" << v[1] << "\t" << v[2] << "\t\n";
  }
}

/// "i y_i" per line (export_graph.hpp:13-23)
template <typename T> void exportGraph(T &yy, std::string filename)
{
  std::ofstream out(filename);
  for(int i = 0; i < (int)yy.size(); i++)
    out << i << " " << yy[i] << "\n";
}

/// one "x y" line; isFirst == 1 recreates the file (export_graph.hpp:55-67)
template <typename T1, typename T2> void addPlot(T1 xx, T2 yy, std::string filename, int isFirst)
{
  std::ofstream out(filename, isFirst == 1 ? std::ios::out : std::ios::app);
  out << xx << " " << yy << "\n";
}

} // namespace icarat
