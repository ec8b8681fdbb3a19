#pragma once
namespace medyan { template <class T> struct BranchingDihedral { static const int n = 4; }; }
