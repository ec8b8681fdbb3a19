#pragma once
namespace medyan { template <class T> struct BranchingBending { static const int n = 4; }; }
