// Build-time generator of shape_tables.inc: the reference-element shape derivatives at the
// quadrature points and the quadrature weights of every element type, as compile-time
// constants for the kernels (exact hexadecimal floats).  Zero entries then fold away.
#include <cstdio>

#include "host.hpp"

int main() {
    std::printf("// generated by gen_tables.cpp from shape.cpp; do not edit\n#pragma once\n");
    std::printf("#ifndef __CUDACC__\n#define __host__\n#define __device__\n#endif\nnamespace octb {\n");
    std::printf("template <int E> struct ShapeConst;\n");
    for (int e : {3, 6, 7, 8, 9}) {
        octb::ShapeTable s;
        octb::shape_table(e, s);
        std::printf("template <> struct ShapeConst<%d> {\n", e);
        std::printf("  __host__ __device__ static constexpr float dN(int k) {\n    constexpr float v[%zu] = {", s.dN.size());
        for (size_t k = 0; k < s.dN.size(); ++k) std::printf("%s%af", k ? "," : "", (float)s.dN[k]);
        std::printf("};\n    return v[k];\n  }\n");
        std::printf("  __host__ __device__ static constexpr float w(int q) {\n    constexpr float v[%d] = {", s.nq);
        for (int q = 0; q < s.nq; ++q) std::printf("%s%af", q ? "," : "", (float)s.w[q]);
        std::printf("};\n    return v[q];\n  }\n};\n");
    }
    std::printf("}  // namespace octb\n");
    return 0;
}
