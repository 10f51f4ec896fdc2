#pragma once
#include "petscsys_shim.h"
