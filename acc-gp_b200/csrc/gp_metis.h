// Host-side METIS step of the V-cycle (see gp_metis.cpp).
#pragma once
#include "gp_internal.h"

#include <cstdint>
#include <string>
#include <vector>

namespace gp {

struct HostCsr {
    int64_t n = 0;
    std::vector<int> off, nbr;
    std::vector<uint32_t> ew, vw;  // materialised (unit weights expanded)
};

gp_status metis_initial_partition(const HostCsr& coarsest, int parts, double eps, uint32_t seed,
                                  std::vector<int>& labels, std::string& error);

}  // namespace gp
