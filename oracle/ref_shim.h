/*
 * TEST INFRASTRUCTURE (the checker, never the product).
 *
 * Lets the reference's OpenCL C kernel source (src/lib.cl of djbarker/boltzmann)
 * compile unmodified as C++. Each OpenCL work-item becomes one plain function call;
 * the work-item id is read from a thread-local array that the host loop in
 * ref_driver.cpp sets before every call.
 */
#pragma once
#include <cmath>
#include <cstddef>
#include <math.h>

#define kernel static
#define global
#define __constant const

static thread_local size_t ref_work_item_id[3];

static inline size_t get_global_id(int dim) { return ref_work_item_id[dim]; }
