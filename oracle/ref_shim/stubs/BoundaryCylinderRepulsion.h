#pragma once
namespace medyan { template <class T> struct BoundaryCylinderRepulsion { static const int n = 1; }; }
