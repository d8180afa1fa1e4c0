/*
 * TEST INFRASTRUCTURE ONLY.  Force-included when the reference's benchmark
 * driver JMSBench1 is compiled (oracle/Makefile, targets jmsbench1-ref and
 * jmsbench1-b200).  test/JMSBench1/prm_main.cpp:57 calls GetGPUCores, whose
 * declaration is commented out in the reference's flat interface
 * (src/JMultiSliceLib.h:213) and which no reference source defines; this
 * declares it so the driver compiles, and gpu_cores.cpp defines it.
 */
#pragma once
int GetGPUCores(int idev, int& nMultiProc, int& nCores, int& nMaxThreadPerProc);
