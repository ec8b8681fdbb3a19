#pragma once
namespace medyan { template <class T> struct CylinderExclVolume { static const int n = 4; }; }
