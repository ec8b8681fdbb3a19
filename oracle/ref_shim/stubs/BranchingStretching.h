#pragma once
namespace medyan { template <class T> struct BranchingStretching { static const int n = 3; }; }
