// Minimal GoogleTest-compatible harness (TEST, TEST_F, EXPECT_* / ASSERT_*,
// testing::internal::CaptureStdout) -- just enough to compile the reference's
// own unit and integration test sources unchanged against libstencil_b200.
// GoogleTest itself is not available in this build environment.
#pragma once

#include <unistd.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace testing {

class Message {
public:
    template <typename T>
    Message& operator<<(const T& v) {
        ss_ << v;
        return *this;
    }
    std::string str() const { return ss_.str(); }

private:
    std::ostringstream ss_;
};

class Test {
public:
    virtual ~Test() = default;
    void RunTest() {
        SetUp();
        TestBody();
        TearDown();
    }

protected:
    virtual void SetUp() {}
    virtual void TearDown() {}
    virtual void TestBody() = 0;
};

namespace internal {

struct TestEntry {
    std::string suite, name;
    std::function<Test*()> make;
};

inline std::vector<TestEntry>& registry() {
    static std::vector<TestEntry> r;
    return r;
}

inline int& failures_in_current_test() {
    static int n = 0;
    return n;
}

struct Registrar {
    Registrar(const char* suite, const char* name, std::function<Test*()> make) {
        registry().push_back({suite, name, std::move(make)});
    }
};

inline void report(const char* file, int line, const std::string& what, const std::string& msg) {
    ++failures_in_current_test();
    std::fprintf(stderr, "%s:%d: Failure\n%s\n%s\n", file, line, what.c_str(), msg.c_str());
}

struct NonFatal {
    const char* file;
    int line;
    std::string what;
    void operator=(const Message& m) const { report(file, line, what, m.str()); }
};

struct Fatal {
    const char* file;
    int line;
    std::string what;
    void operator=(const Message& m) const { report(file, line, what, m.str()); }
};

template <typename T, typename = void>
struct Printable : std::false_type {};
template <typename T>
struct Printable<T, std::void_t<decltype(std::declval<std::ostream&>() << std::declval<const T&>())>>
    : std::true_type {};

template <typename T>
std::string show(const T& v) {
    if constexpr (Printable<T>::value) {
        std::ostringstream s;
        s.precision(17);
        s << v;
        return s.str();
    } else {
        return "<unprintable>";
    }
}

struct Result {
    bool ok;
    std::string text;
    explicit operator bool() const { return ok; }
};

template <typename A, typename B, typename Op>
Result compare(const char* expr, const A& a, const B& b, Op op) {
    if (op(a, b)) return {true, {}};
    return {false, std::string("Expected: ") + expr + "\n  left: " + show(a) + "\n  right: " + show(b)};
}

inline Result near(const char* expr, double a, double b, double tol) {
    if (std::fabs(a - b) <= tol) return {true, {}};
    std::ostringstream s;
    s.precision(17);
    s << "Expected: " << expr << "\n  difference " << std::fabs(a - b) << " exceeds " << tol
      << " (" << a << " vs " << b << ")";
    return {false, s.str()};
}

// Equal within 4 units in the last place, as GoogleTest's FLOAT_EQ / DOUBLE_EQ.
template <typename F, typename U>
bool ulp_equal(F a, F b) {
    if (std::isnan(a) || std::isnan(b)) return false;
    U ua, ub;
    std::memcpy(&ua, &a, sizeof(F));
    std::memcpy(&ub, &b, sizeof(F));
    const U sign = U(1) << (sizeof(U) * 8 - 1);
    auto biased = [sign](U u) { return (u & sign) ? ~u + 1 : (u | sign); };
    const U x = biased(ua), y = biased(ub);
    return (x > y ? x - y : y - x) <= 4;
}

inline Result float_eq(const char* expr, float a, float b) {
    if (ulp_equal<float, uint32_t>(a, b)) return {true, {}};
    return {false, std::string("Expected (float, 4 ulp): ") + expr + "\n  " + show(a) + " vs " +
                       show(b)};
}

inline Result double_eq(const char* expr, double a, double b) {
    if (ulp_equal<double, uint64_t>(a, b)) return {true, {}};
    return {false, std::string("Expected (double, 4 ulp): ") + expr + "\n  " + show(a) + " vs " +
                       show(b)};
}

// stdout capture through a temporary file (CaptureStdout / GetCapturedStdout).
struct Capture {
    int saved = -1;
    FILE* tmp = nullptr;
};
inline Capture& capture_state() {
    static Capture c;
    return c;
}
inline void CaptureStdout() {
    std::fflush(stdout);
    Capture& c = capture_state();
    c.tmp = std::tmpfile();
    c.saved = dup(fileno(stdout));
    dup2(fileno(c.tmp), fileno(stdout));
}
inline std::string GetCapturedStdout() {
    std::fflush(stdout);
    Capture& c = capture_state();
    dup2(c.saved, fileno(stdout));
    close(c.saved);
    std::string out;
    std::rewind(c.tmp);
    char buf[4096];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, c.tmp)) > 0) out.append(buf, n);
    std::fclose(c.tmp);
    c.tmp = nullptr;
    return out;
}

}  // namespace internal

inline void InitGoogleTest(int*, char**) {}

inline int RunAllTests() {
    int failed = 0, run = 0;
    const char* filter = std::getenv("GTEST_SHIM_FILTER");
    for (auto& t : internal::registry()) {
        const std::string full = t.suite + "." + t.name;
        if (filter && *filter && full.find(filter) == std::string::npos) continue;
        ++run;
        std::printf("[ RUN      ] %s\n", full.c_str());
        std::fflush(stdout);
        internal::failures_in_current_test() = 0;
        Test* obj = t.make();
        try {
            obj->RunTest();
        } catch (const std::exception& e) {
            internal::report(__FILE__, __LINE__, "uncaught exception", e.what());
        } catch (...) {
            internal::report(__FILE__, __LINE__, "uncaught exception", "(unknown type)");
        }
        delete obj;
        const bool ok = internal::failures_in_current_test() == 0;
        failed += ok ? 0 : 1;
        std::printf("[ %8s ] %s\n", ok ? "OK" : "FAILED", full.c_str());
        std::fflush(stdout);
    }
    std::printf("[==========] %d tests ran, %d failed\n", run, failed);
    return failed == 0 ? 0 : 1;
}

}  // namespace testing

#define RUN_ALL_TESTS() ::testing::RunAllTests()

#define SHIM_CLASS_(suite, name) suite##_##name##_ShimTest
#define SHIM_DEFINE_(base, suite, name)                                                   \
    class SHIM_CLASS_(suite, name) : public base {                                        \
    protected:                                                                            \
        void TestBody() override;                                                         \
    };                                                                                    \
    static ::testing::internal::Registrar suite##_##name##_shim_reg(                      \
        #suite, #name, [] { return static_cast<::testing::Test*>(new SHIM_CLASS_(suite, name)); }); \
    void SHIM_CLASS_(suite, name)::TestBody()

#define TEST(suite, name) SHIM_DEFINE_(::testing::Test, suite, name)
#define TEST_F(fixture, name) SHIM_DEFINE_(fixture, fixture, name)

#define SHIM_NONFATAL_(res)                                                               \
    if (const ::testing::internal::Result shim_r_ = (res)) {                              \
    } else                                                                                \
        ::testing::internal::NonFatal{__FILE__, __LINE__, shim_r_.text} = ::testing::Message()
#define SHIM_FATAL_(res)                                                                  \
    if (const ::testing::internal::Result shim_r_ = (res)) {                              \
    } else                                                                                \
        return ::testing::internal::Fatal{__FILE__, __LINE__, shim_r_.text} = ::testing::Message()

#define SHIM_CMP_(a, b, op)                                                               \
    ::testing::internal::compare(#a " " #op " " #b, (a), (b),                             \
                                 [](const auto& x, const auto& y) { return x op y; })

#define EXPECT_EQ(a, b) SHIM_NONFATAL_(SHIM_CMP_(a, b, ==))
#define EXPECT_NE(a, b) SHIM_NONFATAL_(SHIM_CMP_(a, b, !=))
#define EXPECT_LT(a, b) SHIM_NONFATAL_(SHIM_CMP_(a, b, <))
#define EXPECT_LE(a, b) SHIM_NONFATAL_(SHIM_CMP_(a, b, <=))
#define EXPECT_GT(a, b) SHIM_NONFATAL_(SHIM_CMP_(a, b, >))
#define EXPECT_GE(a, b) SHIM_NONFATAL_(SHIM_CMP_(a, b, >=))
#define ASSERT_EQ(a, b) SHIM_FATAL_(SHIM_CMP_(a, b, ==))
#define ASSERT_NE(a, b) SHIM_FATAL_(SHIM_CMP_(a, b, !=))
#define ASSERT_LT(a, b) SHIM_FATAL_(SHIM_CMP_(a, b, <))
#define ASSERT_LE(a, b) SHIM_FATAL_(SHIM_CMP_(a, b, <=))
#define ASSERT_GT(a, b) SHIM_FATAL_(SHIM_CMP_(a, b, >))
#define ASSERT_GE(a, b) SHIM_FATAL_(SHIM_CMP_(a, b, >=))
#define EXPECT_TRUE(c) SHIM_NONFATAL_((::testing::internal::Result{bool(c), "Expected true: " #c}))
#define EXPECT_FALSE(c) SHIM_NONFATAL_((::testing::internal::Result{!bool(c), "Expected false: " #c}))
#define ASSERT_TRUE(c) SHIM_FATAL_((::testing::internal::Result{bool(c), "Expected true: " #c}))
#define ASSERT_FALSE(c) SHIM_FATAL_((::testing::internal::Result{!bool(c), "Expected false: " #c}))
#define EXPECT_NEAR(a, b, t) \
    SHIM_NONFATAL_(::testing::internal::near(#a " ~ " #b, double(a), double(b), double(t)))
#define ASSERT_NEAR(a, b, t) \
    SHIM_FATAL_(::testing::internal::near(#a " ~ " #b, double(a), double(b), double(t)))
#define EXPECT_FLOAT_EQ(a, b) \
    SHIM_NONFATAL_(::testing::internal::float_eq(#a " == " #b, float(a), float(b)))
#define EXPECT_DOUBLE_EQ(a, b) \
    SHIM_NONFATAL_(::testing::internal::double_eq(#a " == " #b, double(a), double(b)))

#define EXPECT_THROW(stmt, exc)                                                           \
    SHIM_NONFATAL_(([&]() -> ::testing::internal::Result {                                \
        try {                                                                             \
            stmt;                                                                         \
        } catch (const exc&) {                                                            \
            return {true, {}};                                                            \
        } catch (...) {                                                                   \
            return {false, "Expected " #stmt " to throw " #exc ", it threw another type"}; \
        }                                                                                 \
        return {false, "Expected " #stmt " to throw " #exc ", it did not throw"};         \
    }()))

#define EXPECT_NO_THROW(stmt)                                                             \
    SHIM_NONFATAL_(([&]() -> ::testing::internal::Result {                                \
        try {                                                                             \
            stmt;                                                                         \
        } catch (...) {                                                                   \
            return {false, "Expected " #stmt " not to throw"};                            \
        }                                                                                 \
        return {true, {}};                                                                \
    }()))
