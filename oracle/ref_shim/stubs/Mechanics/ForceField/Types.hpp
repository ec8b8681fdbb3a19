// Stand-in for Mechanics/ForceField/Types.hpp with only EnergyReport, the one
// type the minimizer uses (the real header pulls in Eigen).
#pragma once
#include <string>
#include <vector>
#include "common.h"
namespace medyan {
struct EnergyReport {
    struct EachEnergy { std::string name; floatingpoint energy; };
    floatingpoint total;
    std::vector<EachEnergy> individual;
};
}
