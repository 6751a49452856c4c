// Test infrastructure (oracle only): the reference includes "fresnel.h" (lower case) from
// MicrofacetBeckmann.h while the file on disk is Fresnel.h; this forwards to it.
#pragma once
#include "Fresnel.h"
