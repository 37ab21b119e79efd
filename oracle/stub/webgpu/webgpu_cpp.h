/* Minimal stand-in for the WebGPU C++ header (see webgpu.h in this folder).
 * Only the type names used by the reference's ASTCEncoder declaration exist;
 * none of them can do anything. */
#pragma once
#include "webgpu.h"
namespace wgpu {
struct Device { explicit operator bool() const { return false; } };
struct Queue {};
struct ShaderModule {};
struct ComputePipeline {};
struct BindGroupLayout {};
struct Buffer {};
struct BindGroup {};
}
