#pragma once
namespace medyan {
struct Bead {
    static inline int count = 0;
    static int numBeads() { return count; }
    int getIndex() const { return 0; }
    int getStableIndex() const { return 0; }
};
}
