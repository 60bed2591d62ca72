// Stand-in for the reference's engine/util/Timer.h (which includes SDL_stdinc.h) when
// its CUDA path tracer is compiled on its own for timing on the device. Test
// infrastructure only. CUDAPathTracer::raytrace (cuda_path_tracer.cu:423-464) reads
// Time::totalTime() for its "picture generation time" message; here it is 0.
#pragma once
#include <cstdint>

using Seconds = float;

class Time
{
public:
    static Seconds totalTime() { return 0.0f; }
};
