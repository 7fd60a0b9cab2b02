// Stand-in for VieCut's algorithms.h (VieCut is fetched, not vendored, by the reference).
#pragma once
#include "../../data_structure/mutable_graph.h"
