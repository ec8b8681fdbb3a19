#pragma once
namespace medyan { template <class T> struct BranchingPosition { static const int n = 3; }; }
