// Self-test of the GoogleTest-compatible shim: one passing and three failing
// tests.  The runner must report exactly three failures and exit non-zero.
#include <gtest/gtest.h>

#include <stdexcept>

TEST(ShimSelfTest, Passes) {
    EXPECT_EQ(2 + 2, 4);
    EXPECT_NEAR(1.0, 1.0 + 1e-9, 1e-6);
    EXPECT_FLOAT_EQ(0.1f + 0.2f, 0.3f);
    EXPECT_THROW(throw std::runtime_error("x"), std::runtime_error);
    testing::internal::CaptureStdout();
    std::printf("captured");
    EXPECT_EQ(testing::internal::GetCapturedStdout(), std::string("captured"));
}

TEST(ShimSelfTest, FailsOnCompare) { EXPECT_LT(3, 2) << "planted"; }

TEST(ShimSelfTest, FailsOnNear) { EXPECT_NEAR(1.0, 1.1, 1e-3); }

TEST(ShimSelfTest, FatalStopsTheTest) {
    ASSERT_GT(0, 1);
    EXPECT_TRUE(false);  // not reached: the fatal assertion returned
}
