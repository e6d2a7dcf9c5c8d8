// cukd/kdtree.h -- everything of the drop-in shim (reference cukd/kdtree.h).
#pragma once
#include "cukd/builder.h"
#include "cukd/fcp.h"
#include "cukd/knn.h"
#include "cukd/spatial-kdtree.h"
