#pragma once
namespace medyan { template <class T> struct FilamentStretching { static const int n = 2; }; }
