// Minimal stand-in for googletest (test infrastructure): lets the reference's test sources compile
// so that their checking functions can be called on other data; failed expectations are counted.
#pragma once

#include <exception>

namespace testing
{
struct Test
{
    virtual ~Test() = default;
    virtual void SetUp() {}
    virtual void TearDown() {}
};
} // namespace testing

inline int& ghexref_failures()
{
    static thread_local int n = 0;
    return n;
}
inline void ghexref_expect(bool ok)
{
    if (!ok) ++ghexref_failures();
}

#define EXPECT_TRUE(x) ghexref_expect(static_cast<bool>(x))
#define EXPECT_FALSE(x) ghexref_expect(!static_cast<bool>(x))
#define EXPECT_EQ(a, b) ghexref_expect((a) == (b))
#define EXPECT_NE(a, b) ghexref_expect((a) != (b))
#define EXPECT_NO_THROW(stmt)                                                                                          \
    try                                                                                                                \
    {                                                                                                                  \
        stmt;                                                                                                          \
    }                                                                                                                  \
    catch (...)                                                                                                        \
    {                                                                                                                  \
        ghexref_expect(false);                                                                                         \
    }
#define ASSERT_TRUE(x) EXPECT_TRUE(x)
#define ASSERT_EQ(a, b) EXPECT_EQ(a, b)
#define TEST_F(fixture, name)                                                                                          \
    struct fixture##_##name##_test : fixture                                                                           \
    {                                                                                                                  \
        void TestBody();                                                                                               \
    };                                                                                                                 \
    void fixture##_##name##_test::TestBody()
#define TEST(suite, name) void suite##_##name##_test()
