// Internal hooks between the translation units of libgcz (not part of the C ABI).
#pragma once

#include "gcz.h"

// Records `msg` as the context's last error (under the context lock) and returns `code`.
int gcz_internal_fail(gcz_ctx *c, int code, const char *msg);
