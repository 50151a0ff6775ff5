// Test infrastructure only: entry point for the minimal GoogleTest stand-in.
#include "gtest/gtest.h"

int main() { return mini_gtest::run_all(); }
