#pragma once
namespace medyan { template <class T> struct MotorGhostStretching { static const int n = 4; }; }
