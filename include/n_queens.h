// n_queens.h -- drop-in C++ header for code written against ygch/n_queens.
//
// Same declarations and meaning as the reference's src/n_queens.h for the GPU
// counting path; implemented by libnqueens_b200.so over the C ABI in
// n_queens_b200.h.  The reference's CPU solvers (serial_n_queens,
// parallel_n_queens, n_queens_iterative) are not part of this library: every
// count here runs on the GPU.
#pragma once

#include <vector>

// Whole-board count on one GPU; replaces src/n_queens.h:19 /
// src/n_queens_cuda.cu:84-186.  Prints the reference's progress lines and
// returns 2 x the sum over the half-board prefixes, or -1 when there is no GPU
// (src/n_queens_cuda.cu:105-108).  Any other failure also returns -1 after
// printing the library's error text.
long long cuda_n_queens(int N, int rows);

// Completions of one partial board, added to sum; replaces the per-task
// recursion n_queens() of src/n_queens.h:7 / src/n_queens.cpp:8-21, counted on
// the GPU (the board is split into subtasks and counted in one launch).
void n_queens(int N, int cur, int left, int right, long long &sum);

// Prefix expanders; replace src/n_queens.h:11,13 (src/n_queens.cpp:74-113).
// Append (cur, left, right) int triples to tot, in the reference's order.
void partial_n_queens(int N, int cur, int left, int right, std::vector<int> &tot, int rows);
void partial_n_queens_for_odd(int N, int cur, int left, int right, std::vector<int> &tot, int rows);
