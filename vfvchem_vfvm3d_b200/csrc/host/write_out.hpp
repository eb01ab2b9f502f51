// Field output in the reference's formats (host): ASCII VTK UnstructuredGrid files and CSV lines.
// Every function returns "" on success or the reason it could not write the file.
#pragma once
#include <cstdint>
#include <string>

namespace vfv {

// A field over a tetrahedral mesh's vertices: points, tetrahedra (VTK type 10) and the point data
// array "value" with ncomp (1 or 3) components, or an empty one when values is NULL
// (write_scldom_vtu, src/base/write_vtu.rs:5; write_vecdom_vtu, :192).
std::string write_vtu_tets(const char* path, int64_t n, const double* pos, int64_t ntet, const int32_t* tets, const double* values,
                           int ncomp);

// A field on a vertex set (a boundary's or an interface's nodes): one vertex cell (VTK type 1) per
// vertex (write_sclbnd_vtu, write_sclitf_vtu, write_vecbnd_vtu, write_vecitf_vtu: write_vtu.rs:71,133,259,322).
std::string write_vtu_points(const char* path, int64_t n, const double* pos, const double* values, int ncomp);

// "x,y,z,value" (ncomp 1) or "x,y,z,value_x,value_y,value_z" (ncomp 3) lines after that header
// (src/base/write_csv.rs:5,30,49,68,93,112).
std::string write_csv(const char* path, int64_t n, const double* pos, const double* values, int ncomp);

}  // namespace vfv
