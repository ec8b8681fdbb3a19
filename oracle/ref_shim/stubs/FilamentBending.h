#pragma once
namespace medyan { template <class T> struct FilamentBending { static const int n = 3; }; }
