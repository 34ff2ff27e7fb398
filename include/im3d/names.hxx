/*
 * names.hxx -- common definitions of the header-only API (the reference's
 * header/names.hxx:25-34 defines the same `uint`).
 */
#ifndef IM3D_NAMES_HXX
#define IM3D_NAMES_HXX

#include <cmath>
#include <iostream>
#include <vector>

typedef unsigned int uint;

#endif
