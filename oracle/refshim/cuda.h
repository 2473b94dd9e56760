#pragma once
#include "refshim.h"
