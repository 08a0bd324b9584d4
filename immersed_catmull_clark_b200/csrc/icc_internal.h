// Internal declarations shared by the host set-up (icc_space.cpp) and the device code.
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/icc.h"

namespace icc {

// The four 1-D element matrices of one element: k[0] = int N N, k[1] = int dN N,
// k[2] = int N dN, k[3] = int dN dN (first index = test; rust/src/iga/elasticity.rs:37-58).
struct Mat1d {
    double k[4][3][3];
};

struct Space {
    double lo[3], len[3];
    int64_t nel_dir[3], ncp[3];
    int64_t nel, nsc, ndof;
    std::vector<Mat1d> mats1d[3];  // distinct 1-D matrices per direction
    std::vector<int> type1d[3];    // 1-D type of every element per direction
    // values of the 3 local basis functions of each 1-D type at 3 points of the element:
    // basis1d[d][t][3 i + q] = N_i(x_q), x_q at the Gauss points (same relative points for all)
    std::vector<std::array<double, 9>> basis1d[3];

    bool init(const double bounds[6], const int64_t nsub[3]);
    void element_types(double lambda, double mu, std::vector<double> &ke, std::vector<int32_t> &type_id,
                       std::vector<std::array<int, 3>> &combos) const;
};

int set_error(int code, const std::string &msg);

}  // namespace icc

struct icc_space {
    icc::Space s;
};
