/* Configuration header the reference's CMake would generate (non-MSVC). */
#define IS_MSVC 0
