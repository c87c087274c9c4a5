// Minimal configuration header for building the reference's CPU code path directly
// with g++ (no cmake): every optional third-party backend is switched off.
#pragma once
#ifndef FEAT_CONFIG_HPP
#define FEAT_CONFIG_HPP 1
#define CMAKE_VERSION "none"
#define FEAT_SOURCE_DIR "reference"
#define FEAT_BINARY_DIR "oracle/_ref"
#define BUILD_ID "gcc-opt-serial"
#define FEAT_CPU_TYPE "native"
#define CMAKE_CXX_COMPILER_ID "GNU"
#define FEAT_COMPILER_ID "gcc"
#define CMAKE_CXX_COMPILER_VERSION "13"
#define CMAKE_CXX_COMPILER "g++"
#define CMAKE_CXX_COMPILER_ARG1 ""
#define CMAKE_CXX_COMPILER_ARG1_PATH ""
#define CMAKE_CXX_FLAGS "-O3"
#define FEAT_SYSTEM_HOST_COMPILER "g++"
#define FEAT_CUDA_HOST_COMPILER "g++"
#define FEAT_HOSTNAME "localhost"
#define CMAKE_COMMAND "none"
#define CMAKE_GENERATOR "none"
#define FEAT_GIT_SHA1 "unknown"
#endif
