/* Minimal stand-in for the WebGPU C header, written for this project.
 * The reference's astc.h includes <webgpu/webgpu.h> only to declare its
 * ASTCEncoder class, whose GPU members the oracle never touches.  This file
 * lets the reference's CPU sources (tables, physical packing, .astc store)
 * compile without Dawn. */
#pragma once
#include <stdint.h>
typedef int WGPUCreatePipelineAsyncStatus;
typedef void* WGPUComputePipeline;
