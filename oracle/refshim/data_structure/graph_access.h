// Stand-in for VieCut's graph_access.h (unused by the hot path).
#pragma once
#include "mutable_graph.h"
