"""B200-native (sm_100a) walker propagation and measurement path of miniAFQMC.

  miniafqmc_b200.afqmc      host mirror of the reference operations over the C ABI
  miniafqmc_b200.synthetic  seeded synthetic systems in the reference's data layout
  miniafqmc_b200.driver     the driver loop of miniafqmc_base.cpp on top of the C ABI, with
                            walker sharding, population control and checkpoint / resume
  miniafqmc_b200.build      nvcc build of libafqmc_b200.so and of the driver program
  miniafqmc_b200/miniafqmc  the miniapp's main program over the C ABI (app/miniafqmc.cpp)
"""
