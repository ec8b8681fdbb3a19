#pragma once
#include "ref_stub_counts.h"
namespace medyan {
struct Linker { static CountView<Linker> getLinkers() { return CountView<Linker>{&RefCounts::linkers}; } };
}
