// Stand-in for StreamingUtilities' graph_stream.h (not vendored by the reference).
#pragma once
#include "graph_zeppelin_common.h"
struct GraphStreamUpdate {
  uint8_t type;
  Edge edge;
};
