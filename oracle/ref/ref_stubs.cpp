// Creators of reference objects that the reference oracle does not build:
// they throw when a scene asks for them (test infrastructure).
#include <agz/tracer/create/material.h>

namespace agz::tracer {

// The paper material needs paper_rho_dt.txt, a table the reference checkout
// ships only as a missing large blob.
RC<Material> create_paper(RC<const Texture2D>, real, real, real, real, real, real, real, real, real, real, real,
                          Box<const NormalMapper>) {
    throw ObjectConstructionException("the paper material is not built into the reference oracle");
}

}  // namespace agz::tracer
