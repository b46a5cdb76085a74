// geometry/types.h -- direction and site-parity enums (reference src/geometry/types.h).
#pragma once
enum dir { up, down };
enum site_parity { EV, OD };
