/* Forwarding stand-in for the toolkit header of the same name; see b2e_ref_shim.h. */
#include "b2e_ref_shim.h"
