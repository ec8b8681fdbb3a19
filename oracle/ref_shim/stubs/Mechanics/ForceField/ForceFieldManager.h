// The real ForceFieldManager.h brings Bead and Cylinder into scope for the minimizer.
#pragma once
#include "Bead.h"
#include "Cylinder.h"
