#pragma once
namespace medyan { template <class T> struct LinkerStretching { static const int n = 4; }; }
