// Host edge list behind the opaque plato_edge_list handle (RMAT generator
// and file loader).
#pragma once

#include <vector>

#include "plato_b200.h"

struct plato_edge_list {
  plato_vid_t vertices = 0;
  std::vector<plato_vid_t> src;
  std::vector<plato_vid_t> dst;
  bool weighted = false;
  std::vector<double> w;  // weighted lists: one weight per edge
};
