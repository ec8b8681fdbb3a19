// Timing counters the reference minimizer increments (CUDAcommon::tmin,
// src/Mechanics/CUDAcommon.h:120-281). Only the fields the live minimizer
// code touches are declared; nothing reads them back.
#pragma once
namespace medyan {
struct TimeMinimizationStub {
    double computeenergy = 0, computeenergynonzero = 0, computeenergyzero = 0;
    long computeenerycallsnonzero = 0, computeenerycallszero = 0;
    double computeforces = 0, copyforces = 0, endminimization = 0, findlambda = 0, tother = 0;
};
struct CUDAcommon {
    static inline TimeMinimizationStub tmin;
};
}
