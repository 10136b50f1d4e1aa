// One matching order of a query, seeded with ordered query edge
// (vert[0], vert[1]); shared by the host planner and the device matcher.
#pragma once

#include <cstdint>

namespace dsm {

struct OrderRec {
  uint8_t vert[16];    // query vertex at position p
  uint8_t pos_of[16];  // position of query vertex k
  uint16_t bn[16];     // positions < p adjacent to vert[p] (full query)
};
static_assert(sizeof(OrderRec) == 64, "order record is 64 bytes");

}  // namespace dsm
