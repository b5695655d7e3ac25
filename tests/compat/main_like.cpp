// A driver in the style of the reference's main.cu (main.cu:9-108), built
// against include/xr_compat.hpp and linked with libxr.so.  It loads a preset,
// makes volumes, reconstructs with XTT::reconstruct and writes the direction
// volume, exactly through the reference's names.
//   usage: main_like <settings.json> <tag> <sinogram.raw> <out_prefix>
#include <xr_compat.hpp>

#include <iostream>

int main(int argc, char **argv) {
    if (argc < 5) return 2;
    try {
        init_params(argv[2], argv[1]);
        Volume<float> sinogram[32];
        for (int i = 0; i < NUM_PROJ_COND; i++) sinogram[i] = Volume<float>(NUM_DETECT_U, NUM_DETECT_V, NUM_PROJ);
        Volume<float> all;
        all.load(argv[3], NUM_DETECT_U, NUM_DETECT_V, (int64_t)NUM_PROJ * NUM_PROJ_COND);
        for (int i = 0; i < NUM_PROJ_COND; i++)
            std::memcpy(sinogram[i].get(), all.get() + (size_t)i * NUM_DETECT_U * NUM_DETECT_V * NUM_PROJ,
                        sizeof(float) * NUM_DETECT_U * NUM_DETECT_V * NUM_PROJ);
        Volume<float> ct[32], md[3];
        for (int k = 0; k < NUM_BASIS_VECTOR; k++) {
            ct[k] = Volume<float>(NUM_VOXEL, NUM_VOXEL, NUM_VOXEL);
            ct[k].forEach([](float) -> float { return 0.01f; });   // main.cu:38-43
        }
        for (auto &e : md) e = Volume<float>(NUM_VOXEL, NUM_VOXEL, NUM_VOXEL);
        Geometry geom(SRC_DETECT_DISTANCE, SRC_OBJ_DISTANCE, DETECTOR_SIZE, NUM_VOXEL, NUM_DETECT_U, NUM_PROJ);
        XTT::reconstruct(sinogram, ct, md, geom, 2, 3, Rotate::CW, Method::MLEM, 1e-3);
        for (int k = 0; k < NUM_BASIS_VECTOR; k++)
            ct[k].save(std::string(argv[4]) + "ct" + std::to_string(k + 1) + ".raw");
        for (int i = 0; i < 3; i++) md[i].save(std::string(argv[4]) + "md" + std::to_string(i + 1) + ".raw");
        Volume<float> ev[3];
        for (auto &e : ev) e = Volume<float>(NUM_VOXEL, NUM_VOXEL, NUM_VOXEL);
        Volume<float> md2[3];
        for (auto &e : md2) e = Volume<float>(NUM_VOXEL, NUM_VOXEL, NUM_VOXEL);
        calcEigenVector(ct, md2, ev, 1, 2, 3);   // host, one voxel
        std::cout << "md(1,2,3) " << md[0](1, 2, 3) << " " << md[1](1, 2, 3) << " " << md[2](1, 2, 3) << " host "
                  << md2[0](1, 2, 3) << " " << md2[1](1, 2, 3) << " " << md2[2](1, 2, 3) << std::endl;
    } catch (const std::exception &e) {
        std::cerr << "error: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
