#pragma once
#include "ref_stub_counts.h"
#include "Bead.h"
namespace medyan {
struct Cylinder {
    static CountView<Cylinder> getCylinders() { return CountView<Cylinder>{&RefCounts::cylinders}; }
    int getId() const { return 0; }
    int getStableIndex() const { return 0; }
    Bead* getFirstBead() const { return nullptr; }
    Bead* getSecondBead() const { return nullptr; }
    void printSelf() const {}
    void adjustedrelativeposition(double, bool) const {}
};
}
