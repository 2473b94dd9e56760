/* CUDA launch qualifiers become plain C++ (refshim.h defines them). */
#pragma once
#include "refshim.h"
