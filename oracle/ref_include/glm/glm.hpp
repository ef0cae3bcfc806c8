// Empty stand-in for <glm/glm.hpp>.  The reference headers pulled in by
// oracle/ref_kat_shim.cpp (types.h, constants_structs.h, kernels.cuh,
// eigen_solver.cu, plasticity.cuh) include GLM but the functions compiled from
// them use no GLM type or function.
