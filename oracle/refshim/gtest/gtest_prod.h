// Stand-in for googletest's gtest_prod.h: the reference headers only use FRIEND_TEST.
#pragma once
#define FRIEND_TEST(test_case_name, test_name)
