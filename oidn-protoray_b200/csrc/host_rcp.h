// Reciprocals of per-material and per-table constants, computed on the host CPU.
//
// The reference's CPU build never divides for rcp(x): it takes the hardware's reciprocal
// estimate and refines it with Newton steps (math/math_avx2.h:11-15, math/math_neon.h:10-17).
// The result can sit an ulp or two away from 1/x -- rcp(1.f) is 0.99999994 on AVX2 -- and the
// energy-compensation terms of rough dielectrics amplify such an ulp in eta by the factor
// 1 / (1 - E_avg), up to ~1e5 at low roughness. Every value the reference derives from a
// constant with rcp (eta of each side of an interface, its reciprocal, the Fresnel averages, the
// bounds of the eta <= 1 table axis) is therefore computed here, once, with the same instruction
// sequence on the same CPU, and handed to the device. Per-hit reciprocals stay exact divisions
// on the device; those differ from the reference's by an ulp without amplification.
#pragma once

namespace prt {

// rcp(x) as the reference's CPU build computes it: the estimate instruction, then one Newton
// step r' = 2r - r^2 x on x86-64 (two refinement steps of the estimate on AArch64); 1/x elsewhere.
float hostRcp(float x);

// fresnelDielectricAvg (bsdf/optics.h:137-149): Kulla and Conty's fit of the hemispherical
// average of the dielectric Fresnel reflectance, in the reciprocal of eta taken with hostRcp.
float hostFresnelDielectricAvg(float eta);

} // namespace prt
