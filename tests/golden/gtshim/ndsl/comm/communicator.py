class Communicator:
    pass
