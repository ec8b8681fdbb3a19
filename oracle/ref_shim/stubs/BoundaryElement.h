// Plane boundary element used by the reference boundary-repulsion kernel.
// The reference calls the virtual distance()/normal() of each element in
// BoundaryElement::getBoundaryElements(); this stand-in keeps one global list
// of planes a*x + b*y + c*z + d = 0 whose distance is signed and normalised
// by |(a,b,c)|, matching Structure/BoundaryElementImpl.h (PlaneBoundaryElement).
#pragma once
#include <cmath>
#include <vector>
#include "utility.h"
namespace medyan {
struct BoundaryElement {
    floatingpoint a, b, c, d;
    floatingpoint distance(const floatingpoint* p) const {
        return (a * p[0] + b * p[1] + c * p[2] + d) / std::sqrt(std::pow(a, 2) + std::pow(b, 2) + std::pow(c, 2));
    }
    std::vector<floatingpoint> normal(const floatingpoint*) const { return {a, b, c}; }
    static inline std::vector<BoundaryElement*> elements;
    static std::vector<BoundaryElement*>& getBoundaryElements() { return elements; }
};
}
