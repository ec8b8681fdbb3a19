// Interaction counts read by the reference potential kernels through their
// owning Structure classes (e.g. Cylinder::getCylinders().size()). The shim
// sets these before each call so the reference loops run over exactly the
// arrays the caller passes.
#pragma once
#include <vector>
#include <cstddef>
namespace medyan {
struct RefCounts {
    static inline std::size_t cylinders = 0;
    static inline std::size_t linkers = 0;
    static inline std::size_t motors = 0;
    static inline std::size_t branches = 0;
};
// A collection whose size() is a settable count and whose iteration range is
// empty: the live reference kernels only call size(); the diagnostic branches
// that iterate (taken only after a non-finite force) find no objects.
template <class T>
struct CountView {
    const std::size_t* n;
    std::size_t size() const { return *n; }
    T** begin() const { return nullptr; }
    T** end() const { return nullptr; }
    T* operator[](std::size_t) const { return nullptr; }
};
}
