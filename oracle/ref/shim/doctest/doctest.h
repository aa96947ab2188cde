// Test-infrastructure shim: the reference embeds doctest TEST_CASEs in its
// production sources; doctest itself is not installed here. Test bodies are
// compiled as unused static functions and every assertion is discarded.
#pragma once
#define REYN_SHIM_CAT2(a, b) a##b
#define REYN_SHIM_CAT(a, b) REYN_SHIM_CAT2(a, b)
#define TEST_CASE(name)                                                        \
    [[maybe_unused]] static void REYN_SHIM_CAT(reyn_shim_test_, __LINE__)()
#define TEST_CASE_TEMPLATE(name, T, ...)                                       \
    template <typename T>                                                      \
    [[maybe_unused]] static void REYN_SHIM_CAT(reyn_shim_ttest_, __LINE__)()
#define SUBCASE(name) if (true)
#define CHECK(...) ((void)0)
#define CHECK_FALSE(...) ((void)0)
#define REQUIRE(...) ((void)0)
#define CAPTURE(...) ((void)0)
#define MESSAGE(...) ((void)0)
