#pragma once
#include "ref_stub_counts.h"
namespace medyan {
struct MotorGhost { static CountView<MotorGhost> getMotorGhosts() { return CountView<MotorGhost>{&RefCounts::motors}; } };
}
