/* See volk.h: stand-in for VOLK's allocator header (test infrastructure only). */
#include "volk.h"
