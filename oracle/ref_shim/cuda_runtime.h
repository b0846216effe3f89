#include "gvh_ref_shim.h"
