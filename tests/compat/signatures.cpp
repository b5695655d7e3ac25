// Compile-time check that include/xr_compat.hpp exports the reference's entry
// points with the reference's exact types, so code written against the
// reference's headers binds to them unchanged.  Each alias restates one
// declaration of the reference (file:line given); `g++ -fsyntax-only` is the
// test.
#include <xr_compat.hpp>

#include <string>
#include <type_traits>

using VolF = Volume<float>;

// reconstruct/include/reconstruct.cuh:27-28
using IrReconstruct = void (*)(VolF *, VolF *, const Geometry &, int, int, Rotate, Method, float);
static_assert(std::is_same<decltype(&IR::reconstruct), IrReconstruct>::value, "IR::reconstruct");
// reconstruct/include/reconstruct.cuh:42-45
using XttReconstruct = void (*)(VolF *, VolF *, VolF *, const Geometry &, int, int, Rotate, Method, float);
static_assert(std::is_same<decltype(&XTT::reconstruct), XttReconstruct>::value, "XTT::reconstruct");
// reconstruct/include/reconstruct.cuh:54-55
using FiberReconstruct = void (*)(VolF *, VolF *, const Geometry &, int, int, Rotate, Method, float);
static_assert(std::is_same<decltype(&XTT::fiberModelReconstruct), FiberReconstruct>::value,
              "XTT::fiberModelReconstruct");
// reconstruct/include/reconstruct.cuh:36
using FdkReconstruct = void (*)(VolF *, VolF *, const Geometry &, Rotate);
static_assert(std::is_same<decltype(&FDK::reconstruct), FdkReconstruct>::value, "FDK::reconstruct");
// reconstruct/include/reconstruct.cuh:65
using ForwardProjOnly = void (*)(VolF *, VolF *, const Geometry &, Rotate);
static_assert(std::is_same<decltype(&forwardProjOnly), ForwardProjOnly>::value, "forwardProjOnly");
// direction/include/pca.cuh:9-12
using CalcEigenVector = void (*)(const VolF *, VolF *, VolF *, int, int, int);
static_assert(std::is_same<decltype(&calcEigenVector), CalcEigenVector>::value, "calcEigenVector");
using CalcAngleFromMD = void (*)(const VolF *, VolF *, int, int, int);
static_assert(std::is_same<decltype(&calcAngleFromMD), CalcAngleFromMD>::value, "calcAngleFromMD");
using DirectionNormalization = void (*)(VolF *);
static_assert(std::is_same<decltype(&directionNormalization), DirectionNormalization>::value,
              "directionNormalization");
// solver/include/tvmin.h:9
using TvMin = void (*)(VolF &, float, float, int);
static_assert(std::is_same<decltype(&totalVariationMinimized), TvMin>::value, "totalVariationMinimized");
// reconstruct/include/quadfilt.h:10
using QuadFilt = void (*)(VolF *, VolF *, float);
static_assert(std::is_same<decltype(&quadlicFormFilterCPU), QuadFilt>::value, "quadlicFormFilterCPU");
// reconstruct/include/params.h:37: init_params(tag) is callable as the reference calls it (the
// settings path is a defaulted second argument here)
static_assert(std::is_same<decltype(init_params(std::string())), void>::value, "init_params(tag)");
// the reference's defaulted lambda (reconstruct.cuh:28, :45, :55): calls without it compile
static_assert(std::is_same<decltype(XTT::fiberModelReconstruct(nullptr, nullptr, std::declval<const Geometry &>(), 1,
                                                               1, Rotate::CW, Method::MLEM)),
                           void>::value,
              "fiberModelReconstruct default lambda");
static_assert(std::is_same<decltype(XTT::reconstruct(nullptr, nullptr, nullptr, std::declval<const Geometry &>(), 1, 1,
                                                     Rotate::CW, Method::MLEM)),
                           void>::value,
              "XTT::reconstruct default lambda");
static_assert(std::is_same<decltype(IR::reconstruct(nullptr, nullptr, std::declval<const Geometry &>(), 1, 1,
                                                    Rotate::CW, Method::MLEM)),
                           void>::value,
              "IR::reconstruct default lambda");

int main() { return 0; }
