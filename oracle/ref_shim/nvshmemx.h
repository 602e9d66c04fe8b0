#pragma once
#include "nvshmem.h"
