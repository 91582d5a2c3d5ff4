"""Reconstruction parameters (mirror of dragonfly.params.EMCParams,
dragonfly/params.pyx:9-393) and the INI reader they use (MyConfigParser,
dragonfly/utils/py_src/read_config.py:9-24)."""
import configparser
import os.path as op

RECON3D, RECON2D, RECONRZ = 0, 1, 2
_RTYPES = {"3d": RECON3D, "2d": RECON2D, "rz": RECONRZ}


class MyConfigParser(configparser.ConfigParser):
    """ConfigParser whose file names resolve relative to the config file and
    may point into another section with 'section:::key'."""

    def read(self, filename):
        self.config_folder = op.dirname(filename)
        return super().read(filename)

    def get_filename(self, section, option, *, fallback="NULL"):
        fname = self.get(section, option, fallback=fallback)
        if fname == "NULL":
            raise configparser.NoOptionError(option, section)
        if fname is None or fname == "":
            return fname
        if ":::" in fname:
            subsec, subtag = fname.split(":::")
            fname = self.get_filename(subsec, subtag)
        return op.join(self.config_folder, fname)


class EMCParams:
    """Parameters of an EMC reconstruction, with the reference's defaults
    (params.pyx:13-46) and [emc] keys (params.pyx:67-128)."""

    _FIELDS = ("rank", "num_proc", "iteration", "current_iter", "start_iter", "num_iter", "output_folder",
               "log_fname", "rtype", "save_prob", "verbosity", "beta_period", "need_scaling", "known_scale",
               "update_scale", "alpha", "beta_jump", "beta_factor", "friedel_sym", "axial_sym", "refine",
               "coarse_div", "fine_div", "radius_period", "radius", "radius_jump", "oversampling", "sigmasq",
               "num_modes", "rot_per_mode", "nonrot_modes", "fixed_seed")

    def __init__(self):
        self.rank = 0
        self.num_proc = 1
        self.iteration = 0
        self.current_iter = 0
        self.start_iter = 1
        self.num_iter = 0
        self.known_scale = 0
        self.log_fname = "EMC.log"
        self.output_folder = "data/"
        self.rtype = RECON3D
        self.need_scaling = 0
        self.alpha = 0.
        self.beta_factor = -1.
        self.radius = 0.
        self.num_modes = 1
        self.nonrot_modes = 0
        self.rot_per_mode = 0
        self.beta_jump = 1.
        self.beta_period = 100
        self.radius_jump = 0.
        self.radius_period = 100
        self.oversampling = 10.
        self.sigmasq = 0.
        self.friedel_sym = 0
        self.axial_sym = 1
        self.save_prob = 0
        self.update_scale = 1
        self.refine = 0
        self.coarse_div = 0
        self.fine_div = 0
        self.fixed_seed = 0
        self.verbosity = 0

    def free(self):
        pass

    def from_config(self, config_fname, section_name="emc"):
        config = MyConfigParser()
        config.read(config_fname)
        try:
            self.output_folder = config.get_filename(section_name, "output_folder", fallback="data/")
        except configparser.NoOptionError:
            self.output_folder = "data/"
        try:
            self.log_fname = config.get_filename(section_name, "log_file", fallback="EMC.log")
        except configparser.NoOptionError:
            self.log_fname = "EMC.log"
        rtype = config.get(section_name, "recon_type", fallback="3d")
        if rtype not in _RTYPES:
            raise ValueError("Unknown recon_type %s" % rtype)
        self.rtype = _RTYPES[rtype]
        self.verbosity = config.getint(section_name, "verbosity", fallback=9)
        self.need_scaling = config.getint(section_name, "need_scaling", fallback=0)
        self.alpha = config.getfloat(section_name, "alpha", fallback=0.)
        self.beta_factor = config.getfloat(section_name, "beta_factor", fallback=1.)
        self.radius = config.getfloat(section_name, "radius", fallback=0.)
        self.num_modes = config.getint(section_name, "num_modes", fallback=1)
        self.nonrot_modes = config.getint(section_name, "num_nonrot_modes", fallback=0)
        self.rot_per_mode = config.getint(section_name, "num_rot", fallback=0)
        jump, period = config.get(section_name, "beta_schedule", fallback="1. 100").split()[:2]
        self.beta_jump = float(jump)
        self.beta_period = int(period)
        rj, rp = config.get(section_name, "radius_schedule", fallback="0. 100").split()[:2]
        self.radius_jump = float(rj)
        self.radius_period = int(rp)
        self.oversampling = config.getfloat(section_name, "oversampling", fallback=10.)
        self.sigmasq = config.getfloat(section_name, "gaussian_sigma", fallback=0.) ** 2
        self.friedel_sym = config.getint(section_name, "friedel_sym", fallback=0)
        self.axial_sym = config.getint(section_name, "axial_sym", fallback=1)
        self.save_prob = config.getint(section_name, "save_prob", fallback=0)
        self.update_scale = config.getint(section_name, "update_scale", fallback=1)
        num_divs = config.get(section_name, "num_div", fallback="0").split()
        if len(num_divs) > 1:
            self.refine = 1
            self.fine_div = int(num_divs[0])
            self.coarse_div = int(num_divs[1])
            print("Doing refinement from num_div = %d -> %d\n" % (self.coarse_div, self.fine_div))
        self.fixed_seed = config.getint(section_name, "fixed_seed", fallback=0)

    def __repr__(self):
        return "EMCParams(%s)" % ", ".join("%s=%r" % (k, getattr(self, k)) for k in self._FIELDS)
