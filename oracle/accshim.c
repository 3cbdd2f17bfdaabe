/* Link-time stand-in for acc_set_device_num() used when the reference solver
 * (source/DEM-MPH.cpp:384) is built as a plain OpenMP CPU program with g++:
 * GCC's libgomp aborts on the `acc_device_nvidia` device type, and on the CPU
 * build there is no device to select.  Linked with -Wl,--wrap=acc_set_device_num.
 * Test infrastructure only. */
void __wrap_acc_set_device_num(int num, int type)
{
    (void)num;
    (void)type;
}
