// The caching allocator is not used by the oracle build (CACHE_ALLOC unset).
#pragma once
