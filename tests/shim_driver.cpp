// shim_driver.cpp -- a driver written the way the reference's Landau app drives its plugin
// classes (apps/LandauGaugeFixingSU3_4D.cu:119-271: orStep pairs, projectSU3 every `reproject`
// sweeps, GaugeFixingStats every `checkprecision` sweeps, break below `precision`), compiled
// against include/gfix_culgt.hpp instead of the reference headers.  Used by tests/test_shim.py.
//
//   shim_driver <in.bin> <out.bin> <ormaxiter> <precision> <checkprecision> <reproject>
// in.bin / out.bin: the GpuPattern field (V*72 reals of real_t).  Prints "sweeps gff dA".
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <cuda_runtime.h>

#include "gfix_culgt.hpp"

using gfix_culgt::real_t;

int main(int argc, char **argv)
{
    if (argc != 7) return 2;
    const int Ndim = 4, Nc = 3;
    const short SIZE[4] = {_T_, _X_, gfix_culgt::kNy, gfix_culgt::kNz};
    const long V = (long)SIZE[0] * SIZE[1] * SIZE[2] * SIZE[3];
    const long arraySize = V * Ndim * Nc * Nc * 2;
    std::vector<real_t> U(arraySize);
    FILE *f = std::fopen(argv[1], "rb");
    if (!f || std::fread(U.data(), sizeof(real_t), arraySize, f) != (size_t)arraySize) return 3;
    std::fclose(f);
    const int orMaxIter = std::atoi(argv[3]);
    const double precision = std::atof(argv[4]);
    const int checkPrecision = std::atoi(argv[5]), reproject = std::atoi(argv[6]);

    real_t *dU = nullptr;
    if (cudaMalloc(&dU, arraySize * sizeof(real_t)) != cudaSuccess) return 4;
    cudaMemcpy(dU, U.data(), arraySize * sizeof(real_t), cudaMemcpyHostToDevice);
    const int threadsPerBlock = 8 * 32, numBlocks = (int)(V / 2 / 32);
    GaugeFixingStats<Ndim, Nc, LandauKernelsSU3, 1> gaugeStats(dU, SIZE);
    int sweeps = 0;
    for (int i = 0; i < orMaxIter; i++) {
        LandauKernelsSU3::orStep(numBlocks, threadsPerBlock, dU, nullptr, 0, 1.7f);
        LandauKernelsSU3::orStep(numBlocks, threadsPerBlock, dU, nullptr, 1, 1.7f);
        sweeps = i + 1;
        if (i % reproject == 0) CommonKernelsSU3::projectSU3((int)(V / 32), 32, dU, nullptr);
        if (i % checkPrecision == 0) {
            gaugeStats.generateGaugeQuality();
            if (gaugeStats.getCurrentA() < precision) break;
        }
    }
    CommonKernelsSU3::projectSU3((int)(V / 32), 32, dU, nullptr);
    cudaMemcpy(U.data(), dU, arraySize * sizeof(real_t), cudaMemcpyDeviceToHost);
    cudaFree(dU);
    if (gfix_culgt::last_status != GF_OK) return 5;
    f = std::fopen(argv[2], "wb");
    if (!f) return 6;
    std::fwrite(U.data(), sizeof(real_t), arraySize, f);
    std::fclose(f);
    std::printf("%d %.17g %.17g\n", sweeps, gaugeStats.getCurrentGff(), gaugeStats.getCurrentA());
    return 0;
}
