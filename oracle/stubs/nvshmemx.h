/* Empty stand-in: MGXBench's mulmat_kernel.cu includes this header but uses none of it. */
