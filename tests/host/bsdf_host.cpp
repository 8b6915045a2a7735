// Host harness: the device closure (openpbr.cuh) evaluated on the CPU in
// FP32, for n (wo, wi) pairs read from stdin-named files.
//   bsdf_host <tables.bin> <material.bin> <dirs.bin> <exiting> <out.bin>
// dirs.bin: n × (wo xyz, wi xyz) floats; out.bin: n × (f xyz, pdf) floats.
#include "cuda_host_shim.h"
#include "openpbr.cuh"

#include <cstdio>
#include <vector>

using namespace cn;

int main(int argc, char** argv) {
    if (argc != 6) return 1;
    std::vector<float> tables(T_FLOATS);
    FILE* f = std::fopen(argv[1], "rb");
    if (std::fread(tables.data(), 4, T_FLOATS, f) != T_FLOATS) return 1;
    std::fclose(f);
    Material m;
    f = std::fopen(argv[2], "rb");
    if (std::fread(&m, sizeof m, 1, f) != 1) return 1;
    std::fclose(f);
    f = std::fopen(argv[3], "rb");
    std::vector<float> d;
    float buf[6];
    while (std::fread(buf, 4, 6, f) == 6) d.insert(d.end(), buf, buf + 6);
    std::fclose(f);
    bool exiting = argv[4][0] == '1';
    FILE* o = std::fopen(argv[5], "wb");
    for (size_t i = 0; i + 6 <= d.size(); i += 6) {
        float3 wo = make_float3(d[i], d[i + 1], d[i + 2]), wi = make_float3(d[i + 3], d[i + 4], d[i + 5]);
        Closure c = resolve_closure(tables.data(), m, wo, exiting);
        float3 fv = eval_bsdf(c, wi, wo);
        float p = bsdf_pdf(c, wi, wo);
        float rec[4] = {fv.x, fv.y, fv.z, p};
        std::fwrite(rec, 4, 4, o);
    }
    std::fclose(o);
    return 0;
}
