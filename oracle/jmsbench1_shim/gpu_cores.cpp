// TEST INFRASTRUCTURE ONLY: the GetGPUCores that the reference's JMSBench1
// calls (test/JMSBench1/prm_main.cpp:57) but no reference source defines.
// Fills the multiprocessor count and threads per multiprocessor of device
// idev; nCores is the same count (the driver only prints it).
#include <cuda_runtime.h>

int GetGPUCores(int idev, int& nMultiProc, int& nCores, int& nMaxThreadPerProc)
{
	cudaDeviceProp p;
	if (cudaGetDeviceProperties(&p, idev) != cudaSuccess) return 1;
	nMultiProc = p.multiProcessorCount;
	nCores = p.multiProcessorCount;
	nMaxThreadPerProc = p.maxThreadsPerMultiProcessor;
	return 0;
}
