"""B200-native (sm_100a) rigid-body contact pipeline behind the reference engine's
Backend / C ABI. The compute path is libvelox_b200.so (include/velox_b200.h);
this package only binds it."""
from .binding import (BODY, CONTACT, SPEC, Context, SolverOptions, VeloxError, bodies_from_specs,
                      generate_scene, lib, make_soup)

__all__ = ["BODY", "CONTACT", "SPEC", "Context", "SolverOptions", "VeloxError", "bodies_from_specs",
           "generate_scene", "lib", "make_soup"]
