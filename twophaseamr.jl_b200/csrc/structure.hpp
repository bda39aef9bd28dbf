// Block-structured form of a level (see structure.cpp).
#pragma once

#include <cstdint>
#include <vector>

#include "host.hpp"

namespace tpa {

struct StructLevel {
    int nx = 16, ny = 16;
    int64_t nblocks = 0;
    std::vector<int32_t> nbr;  // 4 per block: W, E, S, N same-size neighbour block or -1
    std::vector<double> cx, cy;  // east / north face coefficients (-a_ij) per cell
    bool const_coef = false;     // every stencil coefficient equals c0 (to 1e-13)
    double c0 = 0;
    std::vector<double> dinv;    // smoother inverse diagonal per cell
    bool const_diag = false;
    bool tinv_same = true;       // the transfer's inverse diagonal equals dinv
    std::vector<int32_t> ex;     // per cell: exception row index or -1
    std::vector<int64_t> ex_ptr; // exception rows (assembled CSR rows)
    std::vector<int32_t> ex_col;
    std::vector<double> ex_val;
    int64_t nex = 0;
    bool has_map = false;        // block map of the tentative transfer is valid
    std::vector<int32_t> map;    // 4 per block: coarse block, x offset, y offset, scale
};

StructLevel build_struct(const HostLevel& lev, const Mesh* coarse_mesh);

}  // namespace tpa
