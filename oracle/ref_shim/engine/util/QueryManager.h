// Host-build stand-in for the reference's engine/util/QueryManager.h.
//
// The reference's LBVH builder (source/application/cuda/BVHBuilder.cu:214,268) wraps
// its work in a CPU timer through QueryManager, whose real header pulls in the
// OpenGL timer-query machinery. For the host build of the reference used as a
// test oracle only the call signatures matter, so the timer is a no-op.
#pragma once
#include <string>

enum class QueryTarget { CPU, GPU };

struct QueryManager {
    static void beginElapsedTime(QueryTarget, const std::string&) {}
    static void endElapsedTime(QueryTarget, const std::string&) {}
};
