// Stand-in for EnTT's entity header, which the reference renderer's shared
// data-structure header includes without using anything from it.  TEST
// INFRASTRUCTURE ONLY (see oracle/ref_shim/sycl/sycl.hpp).
#pragma once
namespace entt {}
