// Stand-in for the reference's HairModel.h in this test build only: the hair
// model (discrete elastic rods) is not part of the liquid step and its
// sources need the full Eigen library, which this machine does not have.
// Scene<3> constructs and owns one; nothing here calls it.
#pragma once

#include "Scene.h"

template <int DIM>
class HairModel {
public:
    explicit HairModel(const Scene<DIM>&) {}
};
