// agz-utils compatibility shim: see _shim.h.
#pragma once
#include "_shim.h"
