#pragma once
#include "ref_stub_counts.h"
namespace medyan {
struct BranchingPoint { static CountView<BranchingPoint> getBranchingPoints() { return CountView<BranchingPoint>{&RefCounts::branches}; } };
}
