// kw_tmaps.cpp — TMA tensor maps of one simulation's spectra for the warp-specialised in-place
// column passes (kw_pass_colp.cu).
//
// Layout axis A (3D only): the half spectrum [A][B][Cp] seen as a 2D tensor [A][B*Cp]; a tile is a
// box of colr_lines(A) consecutive columns by all A rows. Layout axis B: the 3D tensor [A][B][Cp];
// a tile is colr_lines(B) columns of one plane by all B rows (columns past Cp read as zeros).
// The driver entry point cuTensorMapEncodeTiled is resolved through the runtime, so the library
// needs no link against libcuda.
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>

#include "kw_engine.h"

namespace kw {

static KwError err(int code, const std::string& m) { return KwError{code, m}; }

static PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// true when the column pass along `layout_axis` runs the TMA-fed kernel for this simulation
bool colp_enabled(const SimHost& h, int layout_axis) {
    if (layout_axis == 0) return h.dim == 3 && has_colp(h.A);
    return h.dim == 3 && has_colp(h.B);
}

void Engine::build_tensor_maps(SimHost& h, SimDev& v) {
    std::vector<CUtensorMap> maps(kNumTmaps);
    std::memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
    auto fn = encode_tiled();
    const bool any = colp_enabled(h, 0) || colp_enabled(h, 1);
    if (any && !fn) throw err(KW_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    auto encode = [&](CUtensorMap* m, const void* base, int layout_axis) {
        const CUtensorMapDataType ty = CU_TENSOR_MAP_DATA_TYPE_INT64;   // one float2 per element
        const cuuint64_t esz = 8;
        cuuint64_t dims[3];
        cuuint64_t strides[2];
        cuuint32_t box[3], estr[3] = {1, 1, 1};
        cuuint32_t rank;
        if (layout_axis == 0) {
            rank = 2;
            dims[0] = (cuuint64_t)h.B * h.Cp;
            dims[1] = (cuuint64_t)h.A;
            strides[0] = dims[0] * esz;
            box[0] = (cuuint32_t)colr_lines(h.A);
            box[1] = (cuuint32_t)h.A;
        } else {
            rank = 3;
            dims[0] = (cuuint64_t)h.Cp;
            dims[1] = (cuuint64_t)h.B;
            dims[2] = (cuuint64_t)h.A;
            strides[0] = dims[0] * esz;
            strides[1] = dims[0] * dims[1] * esz;
            box[0] = (cuuint32_t)colr_lines(h.B);
            box[1] = (cuuint32_t)h.B;
            box[2] = 1;
        }
        const CUresult r = fn(m, ty, rank, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
            throw err(KW_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ") for a " +
                                       std::to_string(h.A) + "x" + std::to_string(h.B) + "x" + std::to_string(h.Cp) +
                                       " spectrum view");
    };
    for (int axis = 0; axis < 2; ++axis) {
        if (!colp_enabled(h, axis)) continue;
        for (int s = 0; s < 4; ++s)
            if (v.spec[s]) encode(&maps[tmap_spec(s, axis)], v.spec[s], axis);
    }
    // Called twice (before the setup's smoothing jobs and at the end); the contents do not change.
    if (v.tmaps)
        check(cudaMemcpyAsync(const_cast<CUtensorMap*>(v.tmaps), maps.data(), maps.size() * sizeof(CUtensorMap),
                              cudaMemcpyHostToDevice, st()),
              "upload tensor maps");
    else
        v.tmaps = upload(maps);
}

}  // namespace kw
