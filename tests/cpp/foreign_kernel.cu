// A module that is not a handler module: loading it as one must be refused.
extern "C" __global__ void foreign_kernel(int* p) {
  if (p) *p = 1;
}
